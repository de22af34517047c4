"""TEST INFRASTRUCTURE ONLY — FP64 NumPy oracle of jaxdd's transient with mobile ions.

A CPU restatement of `transient.solve_transient` (jaxdd src/jaxdd/transient.py:270-465, 537-637)
for the product's scope: each time step one Newton solve of implicit Euler with the ions as
unknowns of their own (`V, ln n, ln p, ln a, ln c` per point, solver.py:1364-1475
`_assemble_ions`), each region's rescaling a slot of the bordered system (solver.py:1349-1361
`_ion_constraints_time`), the bulk and interface traps' occupations carried from step to step
and solved exactly over each step (solver.py:594-614 `_trap_step`), the current with each
density's change, the ions' currents and the displacement current (batch.py:302-469), and
ZimT's main loop (which steps are kept, `failureMode`, each step's Δt from the last kept one).
Vectorised over a batch of devices of one grid size, as the reference's `vmap`; nothing in the
product imports it.

Scope (the rest is refused, never approximated): the voltage given at every step, or the
internal voltage an unknown of each step (the open circuit, a series resistance); ZimT's
automatic stop (`Track` 2, 3); no photon recycling, no free ends, no ion sites, the steady
scope of `oracle.dd` otherwise. An ion region that reaches a contact takes the
contact's density from its neighbour (`ion_full`). With no mobile ions the same 5-column system
holds the ions' rows at 0 (identity rows); the solution is the reference's 3-column one.

Derivatives that the reference takes by `jax.jvp` (the ions' rows, the traps over a step) are
written out by hand; they are exact, as autodiff is.

Pinning: ZimT 5.36's own transients under the reference's tests/data (`zimt_*`), at the
reference's tolerances (tests/test_transient_oracle.py).
"""

from __future__ import annotations

import numpy as np

from oracle import dd

Q = dd.Q
ION_LOG_CAP = dd.ION_LOG_CAP
STOP_STATIC, STOP_FAILED = 1, 2  # transient.py:240
MIN_COUNT_STATIC = 5  # transient.py:238


def _col(v):
    return np.asarray(v)[:, None]


# ----------------------------------------------------------------------------- traps in time

def trap_step(Cn, Cp, nt0, pt0, n, p, f_old, dti):
    """solver._trap_step (solver.py:594-614) with `empty`: a level's occupation over a step of
    `1/dti` from `f_old`, `df/dt = b − a·f` solved exactly with the densities at the step's end.
    Returns `(mean, end, vacant)` and their derivatives in `n` and in `p`:
    `((mean, end, vacant), (d_n...), (d_p...))`. `dti` broadcasts against the arrays."""
    a = Cn * (n + nt0) + Cp * (p + pt0)
    pos = a > 0
    a = np.where(pos, a, 1.0)
    da_n, da_p = np.where(pos, Cn, 0.0), np.where(pos, Cp, 0.0)
    steady = (Cn * n + Cp * pt0) / a
    vac_s = (Cn * nt0 + Cp * p) / a
    ds_n, ds_p = (Cn - steady * da_n) / a, -steady * da_p / a
    dv_n, dv_p = -vac_s * da_n / a, (Cp - vac_s * da_p) / a
    dti = np.broadcast_to(dti, a.shape)
    moving = dti > 0
    safe = np.where(moving, dti, 1.0)
    x = a / safe
    E = np.where(moving, np.exp(-x), 0.0)
    m = np.where(moving, -np.expm1(-x) / x, 0.0)
    dm = np.where(moving, (E - m) / x, 0.0)       # d m / d x
    dx_n, dx_p = np.where(moving, da_n / safe, 0.0), np.where(moving, da_p / safe, 0.0)
    gap, vgap = f_old - steady, (1.0 - f_old) - vac_s
    mean, end, vac = steady + gap * m, steady + gap * E, vac_s + vgap * m
    d_n = (ds_n * (1.0 - m) + gap * dm * dx_n, ds_n * (1.0 - E) - gap * E * dx_n,
           dv_n * (1.0 - m) + vgap * dm * dx_n)
    d_p = (ds_p * (1.0 - m) + gap * dm * dx_p, ds_p * (1.0 - E) - gap * E * dx_p,
           dv_p * (1.0 - m) + vgap * dm * dx_p)
    return (mean, end, vac), d_n, d_p


def bulk_rates(n, p, r, fb, dti):
    """solver._bulk_rates over a step (solver.py:680-700), one neutral level: each carrier's
    capture by the occupation's mean over the step, `(Rn, Rp)`, and their derivatives in
    `ln n`, `ln p`: `(Rn, Rp, dRn_n, dRn_p, dRp_n, dRp_p)`."""
    Nt, Cn, Cp, nt0, pt0 = r["Nt"], r["Cn"], r["Cp"], r["nt0"], r["pt0"]
    (mean, _, vac), (mn, _, vn), (mp, _, vp) = trap_step(Cn, Cp, nt0, pt0, n, p, fb, dti)
    traps = Nt > 0
    Rn_t = np.where(traps, Nt * Cn * (n * vac - nt0 * mean), 0.0)
    Rp_t = np.where(traps, Nt * Cp * (p * mean - pt0 * vac), 0.0)
    dRn_n = np.where(traps, Nt * Cn * (vac + n * vn - nt0 * mn), 0.0)
    dRn_p = np.where(traps, Nt * Cn * (n * vp - nt0 * mp), 0.0)
    dRp_n = np.where(traps, Nt * Cp * (p * mn - pt0 * vn), 0.0)
    dRp_p = np.where(traps, Nt * Cp * (mean + p * mp - pt0 * vp), 0.0)
    direct = r["kd"] * (n * p - r["ni2"])
    return (direct + Rn_t, direct + Rp_t,
            n * (r["kd"] * p + dRn_n), p * (r["kd"] * n + dRn_p),
            n * (r["kd"] * p + dRp_n), p * (r["kd"] * n + dRp_p))


def bulk_occupation(n, p, r, fb, dti):
    """solver._bulk_occupation (solver.py:711-716): the occupation at the step's end."""
    (_, end, _), _, _ = trap_step(r["Cn"], r["Cp"], r["nt0"], r["pt0"], n, p, fb, dti)
    return end


def iface_edges(nL, nR, pL, pR, ti, f_old, dti):
    """solver._interface_edges over a step (solver.py:814-850, `f_old`): captured by the mean
    occupation, charged by the end's. Values `(Rn_L, Rn_R, Rp_L, Rp_R, Q)` per edge and their
    derivatives in `ln nL, ln nR, ln pL, ln pR` (as `oracle.dd._iface_edges`)."""
    Nt, Cn, Cp, iw = ti["Nt"], ti["Cn"], ti["Cp"], ti["iw"]
    an, bp = Cn * Nt, Cp * Nt
    traps = Nt > 0
    nt0, pt0 = ti["nt0_lo"] + ti["nt0_hi"], ti["pt0_lo"] + ti["pt0_hi"]
    (full, end, empty), (fn, en, vn), (fp, ep, vp) = trap_step(
        Cn, Cp, nt0, pt0, nL + nR, pL + pR, f_old, dti)
    z = np.zeros_like(full)
    full, end, empty = (np.where(traps, v, 0.0) for v in (full, end, empty))
    fn, en, vn, fp, ep, vp = (np.where(traps, v, z) for v in (fn, en, vn, fp, ep, vp))
    half_q = ti["charge"] * 0.5 * Nt * iw
    val = np.stack([iw * an * (nL * empty - ti["nt0_lo"] * full),
                    iw * an * (nR * empty - ti["nt0_hi"] * full),
                    iw * bp * (pL * full - ti["pt0_lo"] * empty),
                    iw * bp * (pR * full - ti["pt0_hi"] * empty),
                    half_q * (ti["cwe"] - end)])
    derivs = []
    for which, dens in enumerate((nL, nR, pL, pR)):
        if which < 2:
            dF, dE, dEnd = fn * dens, vn * dens, en * dens
        else:
            dF, dE, dEnd = fp * dens, vp * dens, ep * dens
        own = [0.0] * 4
        own[which] = 1.0
        derivs.append(np.stack([
            iw * an * (own[0] * nL * empty + nL * dE - ti["nt0_lo"] * dF),
            iw * an * (own[1] * nR * empty + nR * dE - ti["nt0_hi"] * dF),
            iw * bp * (own[2] * pL * full + pL * dF - ti["pt0_lo"] * dE),
            iw * bp * (own[3] * pR * full + pR * dF - ti["pt0_hi"] * dE),
            -half_q * dEnd]))
    return val, derivs


def iface_occupation(n, p, ti, f_old, dti):
    """solver._interface_occupation (solver.py:853-862): each edge's occupation at the step's
    end, on the edges of the full grid."""
    nt0, pt0 = ti["nt0_lo"] + ti["nt0_hi"], ti["pt0_lo"] + ti["pt0_hi"]
    (_, end, _), _, _ = trap_step(ti["Cn"], ti["Cp"], nt0, pt0, n[:, :-1] + n[:, 1:],
                                  p[:, :-1] + p[:, 1:], f_old, dti)
    return np.where(ti["Nt"] > 0, end, 0.0)


def _iface_terms(n, p, ti, f_old, dti):
    """solver._interface_terms (solver.py:876-914) over a step: `(Q, Rn, Rp)` at the interior
    points and their derivatives in the point's own, next and previous `(ln n, ln p)`."""
    val, (d_nL, d_nR, d_pL, d_pR) = iface_edges(n[:, :-1], n[:, 1:], p[:, :-1], p[:, 1:], ti,
                                                f_old, dti)
    lo, hi = [4, 0, 2], [4, 1, 3]
    X = val[hi][:, :, :-1] + val[lo][:, :, 1:]
    own = np.stack([d_nR[hi][:, :, :-1] + d_nL[lo][:, :, 1:],
                    d_pR[hi][:, :, :-1] + d_pL[lo][:, :, 1:]], -1)
    up = np.stack([d_nR[lo][:, :, 1:], d_pR[lo][:, :, 1:]], -1)
    down = np.stack([d_nL[hi][:, :, :-1], d_pL[hi][:, :, :-1]], -1)
    return X, own, up, down


# ----------------------------------------------------------------------------- the system

def assemble(full, d, tr, logs, bern, steady_traps=False, mass=False):
    """solver._assemble_ions (solver.py:1364-1475) with `_assemble`'s carriers' rows over a
    step (solver.py:1021-1187, `tr`; `_bulk_rates` and the interface traps over the step):
    residual F (B×NP×5), blocks A, B, C (B×NP×5×5) and slot columns U (B×NP×5×K) from `full`
    (B×(NP+2)×5). `tr`: `dti` (B), the densities before the step on the interior points
    (`n`, `p`, `a`, `c`, B×NP) and the traps' occupations (`fb` B×NP, `fi` B×(NP+1)).
    `steady_traps`: the traps at their steady occupation (`_time_terms` without occupations,
    as the impedance takes it, impedance.py:251). `mass`: also each row's time term on its own
    unknown per unit of `dti` (B×NP×5; `_assemble_ions(..., mass=True)`)."""
    s, ti, ion = d["s"], d["ti"], d["ion"]
    Vt = _col(d["Vt"])
    dti = _col(tr["dti"])
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
    if steady_traps:
        Rn, dRn_n, dRn_p = dd._recombination(nm, pm, s)
        Rp, dRp_n, dRp_p = Rn, dRn_n, dRn_p
    else:
        Rn, Rp, dRn_n, dRn_p, dRp_n, dRp_p = bulk_rates(nm, pm, s, tr["fb"], dti)
    gen = s["G"] * _col(d["g_frac"])
    dnet_n = np.stack([zm, -dRn_n, -dRn_p], -1)
    dnet_p = np.stack([zm, -dRp_n, -dRp_p], -1)
    elec = hm[..., 0] * Fn[:, 1:] - hp[..., 0] * Fn[:, :-1] + fac * (gen - Rn)
    hole = hp[..., 0] * Fp[:, :-1] - hm[..., 0] * Fp[:, 1:] + fac * (gen - Rp)
    anion = s["a_mask"] * np.exp(full[:, 1:-1, 3])
    cation = s["c_mask"] * np.exp(full[:, 1:-1, 4])
    poisson = (s["fac_l"] * V[:, :-2] + s["fac_m"] * Vm + s["fac_u"] * V[:, 2:]
               - Q * (nm - pm + s["dop"] + s["a_fix"] + anion - s["c_fix"] - cation))
    sP, sC = s["sP"], s["sC"]
    nb, NP = Vm.shape
    A = np.zeros((nb, NP, 5, 5))
    Bb = np.zeros((nb, NP, 5, 5))
    C = np.zeros((nb, NP, 5, 5))
    # Poisson's row: the ions' densities are unknowns of their own, so none follows V.
    A[..., 0, 0] = s["fac_l"] * sP
    C[..., 0, 0] = s["fac_u"] * sP
    Bb[..., 0, 0] = s["fac_m"] * sP
    Bb[..., 0, 1] = -Q * nm * sP
    Bb[..., 0, 2] = Q * pm * sP
    Bb[..., 0, 3] = -Q * anion * sP
    Bb[..., 0, 4] = Q * cation * sP
    A[..., 1, :3] = -hp * dFn0[:, :-1] * sC[..., None]
    A[..., 2, :3] = hp * dFp0[:, :-1] * sC[..., None]
    Bb[..., 1, :3] = (-hp * dFn1[:, :-1] + hm * dFn0[:, 1:] + fac[..., None] * dnet_n) * sC[..., None]
    Bb[..., 2, :3] = (hp * dFp1[:, :-1] - hm * dFp0[:, 1:] + fac[..., None] * dnet_p) * sC[..., None]
    C[..., 1, :3] = hm * dFn1[:, 1:] * sC[..., None]
    C[..., 2, :3] = -hm * dFp1[:, 1:] * sC[..., None]
    if np.any(ti["Nt"] > 0):
        if steady_traps:
            X, own, up, down = dd._iface_terms(n, p, ti)
        else:
            X, own, up, down = _iface_terms(n, p, ti, tr["fi"], dti)
        scale = np.stack([Q * sP, -fac * sC, -fac * sC], 0)  # 3×B×NP
        poisson = poisson + Q * X[0]
        elec = elec - fac * X[1]
        hole = hole - fac * X[2]
        for M, dv in ((A, down), (Bb, own), (C, up)):
            blk = np.moveaxis(dv * scale[..., None], 0, 2)  # B×NP×3×2 in (ln n, ln p)
            M[..., :3, 1:3] += blk
    # implicit Euler in each control volume (ZimT's Cont_Eq_Elec/Holes)
    elec = elec - fac * dti * (nm - tr["n"])
    hole = hole - fac * dti * (pm - tr["p"])
    Bb[..., 1, 1] += -fac * dti * nm * sC
    Bb[..., 2, 2] += -fac * dti * pm * sC
    F = np.zeros((nb, NP, 5))
    F[..., 0], F[..., 1], F[..., 2] = poisson * sP, elec * sC, hole * sC

    # the ions' rows (ZimT's Solve_Neg_Ions, Solve_Pos_Ions; solver.py:1409-1466)
    la_pt, lc_pt = dd.point_logs(logs, ion)
    K = logs.shape[1]
    ka = ion["a_slots"].shape[1]
    U = np.zeros((nb, NP, 5, K))
    ma = ion["a_slots"].sum(1)
    mc = ion["c_slots"].sum(1)
    dti_b = tr["dti"] > 0
    Mass = np.zeros((nb, NP, 5))
    Mass[..., 1] = -fac * nm * sC
    Mass[..., 2] = -fac * pm * sC
    for sn, col, mfull, mu, before, ls, slots, k0 in (
            (-1.0, 3, ma, d["mu_a"], tr["a"], la_pt, ion["a_slots"], 0),
            (1.0, 4, mc, d["mu_c"], tr["c"], lc_pt, ion["c_slots"], ka)):
        m_i = mfull[:, 1:-1]
        el = mfull[:, :-2] * m_i
        el[:, 0] = 0.0
        er = m_i * mfull[:, 2:]
        er[:, -1] = 0.0
        cl, cr = Vt * mu[:, :-2], Vt * mu[:, 1:-1]
        prev = np.where(before > 0, before, 1.0)
        denom = prev * (fac * dti + s["hm"] * cr + s["hp"] * cl)
        scl = 1.0 / np.where(denom != 0, denom, 1.0)  # 0 only outside the regions
        xl = (Vm - V[:, :-2]) / Vt
        xr = (V[:, 2:] - Vm) / Vt
        ll, lcn, lr = full[:, :-2, col], full[:, 1:-1, col], full[:, 2:, col]
        nl, nc, nr = np.exp(ll), np.exp(lcn), np.exp(lr)
        Blf, dBlf = bern(xl)
        Blb, dBlb = bern(-xl)
        Brf, dBrf = bern(xr)
        Brb, dBrb = bern(-xr)
        if sn < 0:  # anions as electrons: F = c·(B(x)·n₁ − B(−x)·n₀)
            Fl, Fr = cl * (Blf * nc - Blb * nl), cr * (Brf * nr - Brb * nc)
            gFl, gFr = cl * (dBlf * nc + dBlb * nl), cr * (dBrf * nr + dBrb * nc)
            flux = er * s["hm"] * Fr - el * s["hp"] * Fl
            dVl = el * s["hp"] * gFl / Vt
            dVc = (-er * s["hm"] * gFr - el * s["hp"] * gFl) / Vt
            dVr = er * s["hm"] * gFr / Vt
            dll = el * s["hp"] * cl * Blb * nl
            dlc = -er * s["hm"] * cr * Brb * nc - el * s["hp"] * cl * Blf * nc
            dlr = er * s["hm"] * cr * Brf * nr
        else:  # cations as holes: F = c·(B(x)·n₀ − B(−x)·n₁)
            Fl, Fr = cl * (Blf * nl - Blb * nc), cr * (Brf * nc - Brb * nr)
            gFl, gFr = cl * (dBlf * nl + dBlb * nc), cr * (dBrf * nc + dBrb * nr)
            flux = el * s["hp"] * Fl - er * s["hm"] * Fr
            dVl = -el * s["hp"] * gFl / Vt
            dVc = (el * s["hp"] * gFl + er * s["hm"] * gFr) / Vt
            dVr = -er * s["hm"] * gFr / Vt
            dll = el * s["hp"] * cl * Blf * nl
            dlc = -el * s["hp"] * cl * Blb * nc - er * s["hm"] * cr * Brf * nc
            dlr = er * s["hm"] * cr * Brb * nr
        els = np.exp(ls)
        moving = (flux + fac * dti * (els * before - nc)) * scl
        steady = lcn - ls + sn * Vm / Vt
        inside = m_i > 0
        mv = inside & dti_b[:, None]
        st = inside & ~dti_b[:, None]
        F[..., col] = np.where(mv, moving, np.where(st, steady, lcn))
        A[..., col, 0] = np.where(mv, dVl * scl, 0.0)
        C[..., col, 0] = np.where(mv, dVr * scl, 0.0)
        A[..., col, col] = np.where(mv, dll * scl, 0.0)
        C[..., col, col] = np.where(mv, dlr * scl, 0.0)
        Bb[..., col, 0] = np.where(mv, dVc * scl, np.where(st, sn / Vt, 0.0))
        Bb[..., col, col] = np.where(mv, (dlc - fac * dti * nc) * scl, 1.0)
        dls = np.where(mv, fac * dti * els * before * scl, np.where(st, -1.0, 0.0))
        kk = slots.shape[1]
        U[..., col, k0:k0 + kk] = dls[..., None] * np.swapaxes(slots[:, :, 1:-1], 1, 2)
        Mass[..., col] = np.where(mv, -fac * nc * scl, 0.0)
    if mass:
        return F, A, Bb, C, U, Mass
    return F, A, Bb, C, U


def constraints(full, logs, ion, dV=None):
    """solver._ion_constraints_time (solver.py:1349-1361): each slot's number of ions over its
    total, less 1, from the ions' own densities (the contacts' from `ion_full`); with its
    derivatives `W` (B×K×NP×5, in each interior point's ion logarithm, and where a region
    reaches a contact in its neighbour's potential through the contact's density, `dV` from
    `ion_full`) and the held slots' identity rows. Returns `(g, W, D)`."""
    masks, totals = dd._masks(ion)
    ka = ion["a_slots"].shape[1]
    nb, K, npts = masks.shape
    col = np.where(np.arange(K) < ka, 3, 4)
    dens = masks * _slot_dens(full, ka, K)
    number = dd._number(dens, masks, ion)
    has = totals > 0
    tot = np.where(has, totals, 1.0)
    held = np.where(has, 0.0, 1.0)
    g = np.where(has, number / tot - 1.0, 0.0) + held * logs
    pair = masks[:, :, 1:] * masks[:, :, :-1] * ion["hL"][:, None, :]
    wpt = 0.5 * (pair[:, :, :-1] + pair[:, :, 1:])
    W = np.zeros((nb, K, npts - 2, 5))
    for k in range(K):
        W[:, k, :, col[k]] = np.where(has[:, k, None], wpt[:, k] * dens[:, k, 1:-1] / tot[:, k, None],
                                      0.0)
        if dV is None:
            continue
        # a contact's density follows its neighbour's ln density and potential
        for side, (c_pt, n_pt, iv) in enumerate(((0, 0, 0), (-1, -1, -1))):
            w = np.where(has[:, k], 0.5 * pair[:, k, iv] * dens[:, k, c_pt] / tot[:, k], 0.0)
            W[:, k, n_pt, col[k]] += w
            W[:, k, n_pt, 0] += w * dV[:, side, col[k] - 3]
    D = np.zeros((nb, K, K))
    D[:, np.arange(K), np.arange(K)] = held
    return g, W, D


def _slot_dens(full, ka, K):
    """Each slot's species' density on every point (B×K×(NP+2)), before the slot's mask."""
    a, c = np.exp(full[..., 3]), np.exp(full[..., 4])
    return np.stack([a if k < ka else c for k in range(K)], 1)


def block_thomas(A, Bb, C, rhs):
    """The block sweep (solver.py:1534-1560) for m×m blocks: rhs B×NP×m×r."""
    nb, NP, m, _ = A.shape
    cp = np.empty_like(C)
    dp = np.empty_like(rhs)
    c_prev = np.zeros_like(C[:, 0])
    d_prev = np.zeros_like(rhs[:, 0])
    for i in range(NP):
        M = Bb[:, i] - A[:, i] @ c_prev
        sol = np.linalg.solve(M, np.concatenate([C[:, i], rhs[:, i] - A[:, i] @ d_prev], -1))
        c_prev, d_prev = sol[..., :m], sol[..., m:]
        cp[:, i], dp[:, i] = c_prev, d_prev
    x = np.empty_like(rhs)
    nxt = np.zeros_like(rhs[:, 0])
    for i in range(NP - 1, -1, -1):
        nxt = dp[:, i] - cp[:, i] @ nxt
        x[:, i] = nxt
    return x


def bordered_solve(A, Bb, C, U, W, D, r, rg):
    """batch._bordered_solve (batch.py:595-603) with `W` on every unknown of a point."""
    X = block_thomas(A, Bb, C, np.concatenate([r[..., None], U], -1))
    XF, XU = X[..., 0], X[..., 1:]
    schur = D - np.einsum("bkir,birl->bkl", W, XU)
    z = np.linalg.solve(schur, (rg - np.einsum("bkir,bir->bk", W, XF))[..., None])[..., 0]
    return XF - np.einsum("birk,bk->bir", XU, z), z


# ----------------------------------------------------------------------------- the current

def width_of(d, zimt):
    """batch._sum_widths (batch.py:406-418): each point's width in the integral form's sum,
    its control volume, or the interval after it with ZimT's sums."""
    NP = d["x"].shape[1] - 2
    hh = d["h"][:, :NP + 1]
    if zimt:
        return hh
    return np.concatenate([hh[:, :1], 0.5 * (hh[:, :-1] + hh[:, 1:])], 1)


def _bern_of(bern, x):
    """`bern`'s B(x); at complex `x` (complex-step derivatives) its analytic continuation."""
    if np.iscomplexobj(x):
        return dd.bern_complex(x, bern is dd.bern_simss)
    return bern(x)[0]


def current(d, full, tr, bern, zimt, steady_traps=False, dU=None, dRi=None):
    """batch._current over a step (batch.py:302-403, 421-483): SIMsalabim's integral form with
    each density's change in the integrand (summed over `width_of`), the ions' currents region
    by region and the displacement current, averaged over the intervals. `tr` as `assemble`'s
    but on the full grid: `dti` (B), `n`, `p`, `a`, `c`, `V` (B×(NP+2)), `fb` (B×NP), `fi`.
    `steady_traps`: the traps at their steady occupation; `dU`, `dRi`: each carrier's rates
    beyond it, bulk and interface, on every point (`tr["dU"]`, `tr["dRi"]`, impedance.py:313).
    Written for complex inputs too (complex-step derivatives), in the integral form."""
    parts, _ = current_parts(d, full, tr, bern, zimt, steady_traps, dU, dRi)
    total = sum(parts.values())
    hh = d["h"][:, :full.shape[1] - 1]
    return np.sum(hh * total, 1) / np.sum(hh, 1)


def current_parts(d, full, tr, bern, zimt, steady_traps=False, dU=None, dRi=None):
    """batch._current_parts over a step (batch.py:316-403): the current's parts on each
    interval (B×(NP+1), SIMsalabim's sign), `Jn`, `Jp`, `Ja`, `Jc`, `JD`, and on the points what
    ZimT's output columns take: `n`, `p`, the generation `gen`, each carrier's recombination `Rn`,
    `Rp` (bulk, the direct included) and interface `Rin`, `Rip`."""
    g_frac = _col(d["g_frac"])
    V, n, p = full[..., 0], np.exp(full[..., 1]), np.exp(full[..., 2])
    Vt, x, h, L = _col(d["Vt"]), d["x"], d["h"], _col(d["L"])
    nb, npts = V.shape
    NP = npts - 2
    dti = _col(tr["dti"])
    if steady_traps:
        Rn = dd._recombination(n, p, d["rec"])[0]
        Rp = Rn
    else:
        pad = np.zeros((nb, 1))
        fb = np.concatenate([pad, tr["fb"], pad], 1)
        Rn, Rp = bulk_rates(n, p, d["rec"], fb, dti)[:2]
    if np.any(d["ti"]["Nt"] > 0):
        if steady_traps:
            val, _ = dd._iface_edges(n[:, :-1], n[:, 1:], p[:, :-1], p[:, 1:], d["ti"])
        else:
            val, _ = iface_edges(n[:, :-1], n[:, 1:], p[:, :-1], p[:, 1:], d["ti"], tr["fi"],
                                 dti)

        def points(lo, hi):
            return np.concatenate([lo[:, :1], hi[:, :-1] + lo[:, 1:], hi[:, -1:]], 1)

        Rin, Rip = points(val[0], val[1]), points(val[2], val[3])
    else:
        Rin = Rip = np.zeros_like(Rn)
    if dU is not None:
        Rn, Rp = Rn + dU[0], Rp + dU[1]
    if dRi is not None:
        Rin, Rip = Rin + dRi[0], Rip + dRi[1]
    dx = np.diff(x[:, :NP + 1], axis=1)
    width = width_of(d, zimt)
    G = d["G"]

    def carrier(sn, Vg, dens, mu, R, R_i, before):
        Uc = R + R_i - G * g_frac
        Uc[:, 0] = 0.0
        Uc[:, -1] = 0.0
        change = dti * (dens - before)
        if not zimt:
            change[:, 0] = 0.0
        Uc = Uc + change
        with np.errstate(over="ignore", invalid="ignore"):
            ev = np.exp(sn * Vg[:, :NP + 1] / Vt)
            int_u = np.concatenate([np.zeros((nb, 1)),
                                    np.cumsum(0.5 * dx * (Uc[:, :NP] + Uc[:, 1:NP + 1]), 1)], 1)
            single = np.sum(0.5 * dx * (ev[:, :-1] / mu[:, :NP] + ev[:, 1:] / mu[:, 1:NP + 1]), 1)
            double = np.sum(0.5 * dx * (ev[:, :-1] * int_u[:, :-1] / mu[:, :NP]
                                        + ev[:, 1:] * int_u[:, 1:] / mu[:, 1:NP + 1]), 1)
            K = (Vt[:, 0] * (sn * dens[:, NP + 1] * np.exp(sn * Vg[:, NP + 1] / Vt[:, 0])
                             - sn * dens[:, 0] * np.exp(sn * Vg[:, 0] / Vt[:, 0]))
                 - sn * double) / single
        J = Q * K[:, None] + np.concatenate(
            [np.zeros((nb, 1)), np.cumsum(sn * Q * L * width[:, 1:NP + 1] * Uc[:, 1:NP + 1], 1)], 1)
        diff = d["curr_diff"] > 0
        if np.any(diff):
            dV = sn * np.diff(Vg, axis=1) / Vt
            Bm, Bp = _bern_of(bern, -dV), _bern_of(bern, dV)
            flux = sn * Q * mu[:, :NP + 1] * Vt * (dens[:, 1:] * Bm - dens[:, :-1] * Bp) / (
                L * h[:, :NP + 1])
            J = np.where(diff[:, None], flux, J)
        through = sn * 0.5 * Q * L * h[:, :NP + 1] * (R_i[:, :NP + 1] + R_i[:, 1:])
        return np.where(d["iface"], np.roll(J, 1, axis=1) + through, J)

    sign = -_col(d["left_elec"])
    Ja, Jc = ion_currents(d, full, tr, bern, width, apart=True)
    parts = {"Jn": sign * carrier(-1.0, V + d["offset_n"], n, d["mu_n"], Rn, Rin, tr["n"]),
             "Jp": sign * carrier(1.0, V + d["offset_p"], p, d["mu_p"], Rp, Rip, tr["p"]),
             "Ja": sign * Ja, "Jc": sign * Jc,
             "JD": sign * d["eps"][:, :NP + 1] * (np.diff(V, axis=1) - np.diff(tr["V"], axis=1))
             * dti / (L * h[:, :NP + 1])}
    points = {"n": n, "p": p, "gen": G * g_frac, "Rn": Rn, "Rp": Rp, "Rin": Rin, "Rip": Rip}
    return parts, points


def ion_currents(d, full, tr, bern, width, apart=False):
    """batch._ion_currents (batch.py:421-483): each region's current over the step from its
    integral form with the densities' change as the integrand; 0 outside, every region's
    counted, or with `tr["ion_last"]` (B, true) each species' last region's alone (ZimT 5.36's
    with several regions). The anions' and cations' summed, on the NP + 1 intervals, or with
    `apart` each species' `(Ja, Jc)`."""
    ion = d["ion"]
    Vt, x, h, L = _col(d["Vt"]), d["x"], d["h"], _col(d["L"])
    V = full[..., 0]
    nb, npts = V.shape
    NP = npts - 2
    dx = np.diff(x, axis=1)
    dti = _col(tr["dti"])
    masks, totals = dd._masks(ion)
    ka = ion["a_slots"].shape[1]
    out = [np.zeros((nb, NP + 1)), np.zeros((nb, NP + 1))]
    e = np.arange(NP + 1)
    idx = np.arange(masks.shape[1])[None]
    last_a = np.max(np.where((totals > 0) & (idx < ka), idx, -1), 1)
    last_c = np.max(np.where((totals > 0) & (idx >= ka), idx, -1), 1)
    only_last = np.asarray(tr.get("ion_last", np.zeros(nb, bool)), bool)
    for k in range(masks.shape[1]):
        anion = k < ka
        sn = -1.0 if anion else 1.0
        dens = np.exp(full[..., 3] if anion else full[..., 4])
        before = tr["a"] if anion else tr["c"]
        mu = d["mu_a"] if anion else d["mu_c"]
        mask = masks[:, k]
        pair = mask[:, 1:] * mask[:, :-1]
        Uc = dti * (dens - before)
        with np.errstate(over="ignore", invalid="ignore"):
            ev = np.exp(sn * V / Vt)
            mu_ = np.where(mu > 0, mu, 1.0)
            int_u = np.concatenate([np.zeros((nb, 1)),
                                    np.cumsum(0.5 * dx * (Uc[:, :-1] + Uc[:, 1:]) * pair, 1)], 1)
            single = np.sum(0.5 * dx * (ev[:, :-1] / mu_[:, :-1] + ev[:, 1:] / mu_[:, 1:]) * pair, 1)
            double = np.sum(0.5 * dx * (ev[:, :-1] * int_u[:, :-1] / mu_[:, :-1]
                                        + ev[:, 1:] * int_u[:, 1:] / mu_[:, 1:]) * pair, 1)
            first = np.argmax(mask > 0, 1)
            last = npts - 1 - np.argmax(mask[:, ::-1] > 0, 1)
            single = np.where(np.real(single) > 0, single, 1.0)
            rows = np.arange(nb)
            ends = sn * (dens[rows, last] * ev[rows, last] - dens[rows, first] * ev[rows, first])
            Kk = (Vt[:, 0] * ends - sn * double) / single
        step = np.where(e[None] > first[:, None], sn * Q * L * width * Uc[:, :NP + 1], 0.0) * pair
        J = Q * Kk[:, None] + np.cumsum(step, 1)
        diff = d["curr_diff"] > 0
        if np.any(diff):
            dV = sn * np.diff(V, axis=1) / Vt
            Bm, Bp = _bern_of(bern, -dV), _bern_of(bern, dV)
            flux = sn * Q * mu[:, :NP + 1] * Vt * (dens[:, 1:] * Bm - dens[:, :-1] * Bp) / (
                L * h[:, :NP + 1])
            J = np.where(diff[:, None], flux, J)
        J = np.where(d["iface"], np.roll(J, 1, axis=1), J)
        counted = (totals[:, k] > 0) & (~only_last | (k == (last_a if anion else last_c)))
        out[0 if anion else 1] = out[0 if anion else 1] + np.where(
            (pair > 0) & counted[:, None], J, 0.0)
    return tuple(out) if apart else out[0] + out[1]


def columns(layers, d, parts, points, full, J, J_ext):
    """transient._columns (transient.py:163-222): ZimT's tJFile columns beyond the voltages and
    currents at one step, per device of the batch (`layers` each device's `(i0, i1)`): `errJ`,
    the current's rms deviation over the grid from its average; per layer the QFLS averaged on
    the grid, the photocurrent and each carrier's direct and bulk recombination as currents
    (`EquiCurr`), and at each layer's right end the interface traps' recombination of each
    carrier; the minority carriers' currents at the contacts, the shunt's, the ions' and the
    displacement current averaged; each layer's voltage drop. Per-layer columns B×(most
    layers), 0 past a device's own."""
    nb, npts = full.shape[:2]
    NP = npts - 2
    x, h, L, Vt = d["x"], d["h"], d["L"], d["Vt"]
    hh = h[:, :NP + 1]
    total = sum(parts.values())
    dev = np.concatenate([total, total[:, -1:]], 1) - _col(J)
    out = {"errJ": np.sqrt(np.sum(dev ** 2, 1) / (NP + 1))}
    nl = max(len(i0) for i0, _ in layers)
    per = {k: np.zeros((nb, nl)) for k in ("QFLS", "Jphoto", "Jdir", "JbulkElec", "JbulkHoles",
                                           "JintElec", "JintHoles", "VL")}
    n, p, V = points["n"], points["p"], full[..., 0]
    ni2 = d["rec"]["ni2"]
    qfls = _col(Vt) * (np.log(n) + np.log(p) - np.log(ni2))
    direct = d["rec"]["kd"] * (n * p - ni2)
    hpad = np.concatenate([h, np.zeros((nb, npts - h.shape[1]))], 1)
    for b, (i0, i1) in enumerate(layers):
        def interior(v):
            v = v.copy()
            v[0] = v[-1] = 0.0
            return v

        for j, (a, e) in enumerate(zip(i0, i1)):
            w = hh[b, a:e]
            norm = np.sum(w) if np.sum(w) > 0 else 1.0

            def average(v):
                return np.sum(w * v[a:e]) / norm

            def equi(v):
                return Q * average(interior(v)) * (x[b, e] - x[b, a])

            per["QFLS"][b, j] = average(0.5 * (qfls[b, :-1] + qfls[b, 1:]))
            per["Jphoto"][b, j] = equi(points["gen"][b])
            per["Jdir"][b, j] = equi(direct[b])
            per["JbulkElec"][b, j] = equi(points["Rn"][b] - direct[b])
            per["JbulkHoles"][b, j] = equi(points["Rp"][b] - direct[b])
            nxt = e + 1 if e + 1 < npts else 0  # `roll`: the point after the layer's last
            per["JintElec"][b, j] = Q * L[b] * hpad[b, e] * (points["Rin"][b, e]
                                                            + points["Rin"][b, nxt])
            per["JintHoles"][b, j] = Q * L[b] * hpad[b, e] * (points["Rip"][b, e]
                                                             + points["Rip"][b, nxt])
            per["VL"][b, j] = V[b, e] - V[b, a]
    out.update(per)

    def mean(v):
        return np.sum(hh * v, 1) / np.sum(hh, 1)

    Jn, Jp = parts["Jn"], parts["Jp"]
    out["JminLeft"] = np.where(n[:, 0] < p[:, 0], Jn[:, 0], Jp[:, 0])
    out["JminRight"] = np.where(n[:, -1] < p[:, -1], Jn[:, -1], Jp[:, -1])
    out["JShunt"] = J_ext - J
    out["Jnion"], out["Jpion"], out["JD"] = mean(parts["Ja"]), mean(parts["Jc"]), mean(parts["JD"])
    return out


# ----------------------------------------------------------------------------- Newton in time

def _caps(Vt):
    return np.stack([dd.STEP_CAPS[0] * Vt] + [np.full_like(Vt, dd.STEP_CAPS[1])] * 4,
                    -1)[:, None, :]


def full_of(d, y, Vint, bern=None, dti=None):
    """`y` (B×NP×5) with the contacts' rows (batch._full, batch.py:262-267); the contacts' ions
    0, or with `bern` and `dti` (B) each region's that reaches a contact (`ion_full`)."""
    bnd = dd.bounds(d, Vint)
    b = np.concatenate([bnd, np.zeros(bnd.shape[:2] + (2,))], -1)
    full = np.concatenate([b[:, :1], y, b[:, 1:]], 1)
    return full if bern is None else ion_full(d, full, bern, dti)[0]


def ion_full(d, full, bern, dti):
    """solver._ion_full (solver.py:1315-1346) without ion sites or free ends: each contact's
    ions where a region reaches it, from its neighbour so that nothing flows over the contact's
    interval (`ln a_0 = ln a_1 + ln(B(x)/B(-x))`, x = (V_1 - V_0)/V_T, the cations' the other
    way; Boltzmann's, the ratio -x, in the steady state `dti = 0`), 0 elsewhere. Returns the
    full state and each contact's ln a, ln c derivative in its neighbour's potential
    (B×2×2: left, right × anion, cation; 0 for a complex `full`, whose contacts' values are
    continued analytically for complex-step derivatives)."""
    ion = d["ion"]
    Vt = d["Vt"]
    ma, mc = ion["a_slots"].sum(1), ion["c_slots"].sum(1)
    V = full[..., 0]
    moving = np.asarray(dti, dtype=float) > 0

    def ratio(x):
        if np.iscomplexobj(x):  # complex-step derivatives: the value alone, continued
            simss = bern is dd.bern_simss
            r = np.log(dd.bern_complex(x, simss)) - np.log(dd.bern_complex(-x, simss))
            return np.where(moving, r, -x), np.zeros(x.shape)
        Bf, dBf = bern(x)
        Bb, dBb = bern(-x)
        with np.errstate(divide="ignore", invalid="ignore"):
            return (np.where(moving, np.log(Bf) - np.log(Bb), -x),
                    np.where(moving, dBf / Bf + dBb / Bb, -1.0))

    r0, dr0 = ratio((V[:, 1] - V[:, 0]) / Vt)
    rN, drN = ratio((V[:, -1] - V[:, -2]) / Vt)
    out = full.copy()
    out[:, 0, 3] = np.where(ma[:, 0] > 0, full[:, 1, 3] + r0, 0.0)
    out[:, 0, 4] = np.where(mc[:, 0] > 0, full[:, 1, 4] - r0, 0.0)
    out[:, -1, 3] = np.where(ma[:, -1] > 0, full[:, -2, 3] - rN, 0.0)
    out[:, -1, 4] = np.where(mc[:, -1] > 0, full[:, -2, 4] + rN, 0.0)
    dV = np.stack([np.stack([dr0, -dr0], -1), np.stack([drN, -drN], -1)], 1) / Vt[:, None, None]
    return out, dV


def newton_step(y, logs, d, Vint, tr, bern):
    """One damped Newton step of a time step (batch.py:759-785 with `_system`'s 5-column form,
    518-530)."""
    full, dV = ion_full(d, full_of(d, y, Vint), bern, tr["dti"])
    F, A, Bb, C, U = assemble(full, d, tr, logs, bern)
    g, W, D = constraints(full, logs, d["ion"], dV)
    delta, d_logs = bordered_solve(A, Bb, C, U, W, D, -F, -g)
    caps = _caps(d["Vt"])
    stepv = dd.density_steps(y, delta, np.clip(delta, -caps, caps), d["s"]["n_floor"])
    d_logs = np.clip(d_logs, -ION_LOG_CAP, ION_LOG_CAP)
    new = y + stepv
    with np.errstate(over="ignore", invalid="ignore"):
        dens = np.exp(new[..., 1:])
        weight = dens / (dens + d["s"]["n_floor"][..., None])
        size = np.maximum(np.maximum(np.max(np.abs(stepv[..., 0]), 1) / d["Vt"],
                                     np.max(np.abs(stepv[..., 1:]) * weight, axis=(1, 2))),
                          np.max(np.abs(d_logs), 1))
    return new, logs + d_logs, size


def newton_step_vint(y, logs, Vint, d, tr, trc, bern, zimt, oc, Vext):
    """One damped Newton step with the internal voltage an unknown (batch._system_vint,
    batch.py:552-592, and the step of _newton_loop, 759-785): its column the rows' derivatives in
    it through the contacts' potentials (`V_0 = V0 + e Vint/2`, `V_N+1 = VL - e Vint/2`), its row
    the external current over the current scale at the open circuit (`oc`), else
    `(Vint + R_series J_ext - Vext)/V_T`. The row's products with the block sweep's solutions
    (dense in the grid) are complex-step derivatives of the current along each solution, exact
    as the reference's `jax.value_and_grad`; its own derivative in Vint the same. Returns the new
    state, slots, voltage and step size."""
    full, dV = ion_full(d, full_of(d, y, Vint), bern, tr["dti"])
    F, A, Bb, C, U = assemble(full, d, tr, logs, bern)
    g, W, D = constraints(full, logs, d["ion"], dV)
    e = d["left_elec"]
    Uv = np.zeros(F.shape)
    Uv[:, 0] += A[:, 0, :, 0] * _col(0.5 * e)
    Uv[:, -1] += C[:, -1, :, 0] * _col(-0.5 * e)
    Vt, R, Js = d["Vt"], d["R_series"], d["J_scale"]
    G_shunt = d["G_shunt"]

    def J_ext(y_, V_):
        return current(d, full_of(d, y_, V_), trc, bern, zimt) + G_shunt * V_

    Je = J_ext(y, Vint)
    h = np.where(oc, Je / Js, (Vint + R * Je - Vext) / Vt)
    coef = np.where(oc, 1.0 / Js, R / Vt)
    X = block_thomas(A, Bb, C, np.concatenate([-F[..., None], U, Uv[..., None]], -1))
    delta = 1e-20
    hX = np.stack([coef * np.imag(J_ext(y + 1j * delta * X[..., c], Vint)) / delta
                   for c in range(X.shape[-1])], -1)
    dJ_dV = np.imag(J_ext(y, Vint + 1j * delta)) / delta
    h_V = np.where(oc, dJ_dV / Js, (1.0 + R * dJ_dV) / Vt)
    K = W.shape[1]
    WX = np.einsum("bkir,birc->bkc", W, X)
    rows = np.concatenate([WX, hX[:, None, :]], 1)  # (K+1) rows × (1 + K + 1) columns
    Dv = np.zeros((y.shape[0], K + 1, K + 1))
    Dv[:, :K, :K] = D
    Dv[:, K, K] = h_V
    schur = Dv - rows[:, :, 1:]
    rg = -np.concatenate([g, h[:, None]], 1) - rows[:, :, 0]
    z = np.linalg.solve(schur, rg[..., None])[..., 0]
    dy = X[..., 0] - np.einsum("birk,bk->bir", X[..., 1:], z)
    caps = _caps(Vt)
    stepv = dd.density_steps(y, dy, np.clip(dy, -caps, caps), d["s"]["n_floor"])
    d_logs = np.clip(z[:, :K], -ION_LOG_CAP, ION_LOG_CAP)
    d_V = np.clip(z[:, K], -dd.STEP_CAPS[0] * Vt, dd.STEP_CAPS[0] * Vt)
    new = y + stepv
    with np.errstate(over="ignore", invalid="ignore"):
        dens = np.exp(new[..., 1:])
        weight = dens / (dens + d["s"]["n_floor"][..., None])
        size = np.maximum(np.maximum(np.max(np.abs(stepv[..., 0]), 1) / Vt,
                                     np.max(np.abs(stepv[..., 1:]) * weight, axis=(1, 2))),
                          np.maximum(np.max(np.abs(d_logs), 1), np.abs(d_V) / Vt))
    return new, logs + d_logs, Vint + d_V, size


def _take_tr(tr, idx):
    return {k: v[idx] for k, v in tr.items()}


def newton_loop(y, logs, d, Vint, tr, trc, bern, tol, max_iter, zimt, vint=None):
    """batch._newton_loop (batch.py:740-848) over a time step: `tr` the step's terms on the
    interior points (`assemble`), `trc` on the full grid (`current`). `vint`: `(oc, Vext)` (B
    each) with the internal voltage an unknown from `Vint` (`newton_step_vint`; the current's
    settling then no stop); returns the voltage too."""
    nb = y.shape[0]
    y, logs = y.copy(), logs.copy()
    Vint = np.array(Vint, dtype=float)
    S = dd.STALL_STEPS
    size_h = np.full((nb, S + 1), np.inf)
    J_h = np.full((nb, S + 1), np.inf)
    it = np.zeros(nb, dtype=int)
    done = np.zeros(nb, bool)
    while True:
        active = ~done & (it < max_iter) & ~np.isnan(size_h[:, -1])
        if not active.any():
            break
        idx = np.flatnonzero(active)
        dl = dd.take(d, idx)
        if vint is None:
            new, logs_new, size = newton_step(y[idx], logs[idx], dl, Vint[idx],
                                              _take_tr(tr, idx), bern)
        else:
            new, logs_new, Vint[idx], size = newton_step_vint(
                y[idx], logs[idx], Vint[idx], dl, _take_tr(tr, idx), _take_tr(trc, idx), bern,
                zimt, vint[0][idx], vint[1][idx])
        J = current(dl, full_of(dl, new, Vint[idx], bern, trc["dti"][idx]), _take_tr(trc, idx),
                    bern, zimt)
        sh = np.concatenate([size_h[idx, 1:], size[:, None]], 1)
        jh = np.concatenate([J_h[idx, 1:], J[:, None]], 1)
        n_it = it[idx] + 1
        size_now, prev = sh[:, -1], sh[:, -2]
        with np.errstate(invalid="ignore"):
            stalled = ((n_it > S) & (np.max(sh, 1) < dd.ROUND_OFF_FLOOR)
                       & (np.min(sh[:, 1:], 1) >= 0.1 * sh[:, 0]))
            scale = dl["J_scale"] + np.abs(jh[:, -1])
            settled = ((n_it > S) & (size_now < dd.CURRENT_STEP_CAP)
                       & (np.max(np.abs(jh - jh[:, -1:]), 1) < dd.CURRENT_TOL * scale))
            quadratic = (n_it > 1) & (size_now < dd.QUADRATIC_TOL) & (
                size_now < dd.QUADRATIC_RATIO * prev)
            if vint is not None:
                settled = np.zeros_like(settled)
            conv = (size_now < tol) | stalled | settled | quadratic
        y[idx], logs[idx] = new, logs_new
        size_h[idx], J_h[idx], it[idx], done[idx] = sh, jh, n_it, conv
    if vint is not None:
        return y, logs, J_h[:, -1], done, it, Vint
    return y, logs, J_h[:, -1], done, it


# ----------------------------------------------------------------------------- the steps

def summary(d, full):
    """What two states compare by (transient.py:361-368) without the current: `V`, `n`, `p`,
    `a`, `c` on every point (B×(NP+2) each, the ions where mobile)."""
    ion = d["ion"]
    ma, mc = ion["a_slots"].sum(1), ion["c_slots"].sum(1)
    return {"V": full[..., 0], "n": np.exp(full[..., 1]), "p": np.exp(full[..., 2]),
            "a": np.exp(full[..., 3]) * ma, "c": np.exp(full[..., 4]) * mc}


def states_equal(A, B, GA, GB, tol_pois, tol_dens, conv_var=1, tol_curr=None, JA=None, JB=None,
                 errA=None, errB=None):
    """ZimT's `States_Are_Equal` (transient.py:243-262): the same `G_frac`, the potentials within
    `tolPois` (V, the Euclidean norm over the grid), then by `convVar` each density relatively
    within `tolDens` (1), the currents `J` within `tolCurr` or the smaller of the two states'
    errJ (2), either (3) or both (4)."""
    def norm(v):
        return np.sqrt(np.sum(v ** 2, axis=1))

    def rel(a, b):
        scale = 0.5 * (norm(a) + norm(b))
        return np.where(scale > 0, norm(a - b) / np.where(scale > 0, scale, 1.0), 0.0)

    dens = np.all(np.stack([rel(A[k], B[k]) for k in ("n", "p", "a", "c")]) < tol_dens, 0)
    cv = np.asarray(conv_var)
    if np.all(cv == 1):
        by = dens
    else:
        curr = np.abs(JA - JB) <= np.maximum(tol_curr, np.minimum(errA, errB))
        by = np.where(cv == 1, dens, np.where(cv == 2, curr, np.where(cv == 3, curr | dens,
                                                                      curr & dens)))
    return (GA == GB) & (norm(A["V"] - B["V"]) < tol_pois) & by


def check_scope(d, oc=None, track=None, conv_var=None):
    """What this restatement (and the product) supports; the rest raises."""
    vint = np.any(d["R_series"] > 0) or (oc is not None and np.any(oc))
    masks, _ = dd._masks(d["ion"])
    if vint and (np.any(masks[:, :, 0] > 0) or np.any(masks[:, :, -1] > 0)):
        raise NotImplementedError("the internal voltage an unknown with an ion region that "
                                  "reaches a contact")


def solve_transient(batch, t, V, G_frac, track=None, failure_mode=1, tol=1e-10, max_iter=200,
                    bernoulli_name="exact", zimt_current=False, zimt_ion_currents=False,
                    oc=None, conv_var=1, tol_pois=1e-6, tol_dens=1e-6, tol_curr=1e-3,
                    layers=None):
    """transient.solve_transient / _solve_one (transient.py:270-465, 537-637) for every lane at
    once. `t`, `V`, `G_frac`, `track`: (S,) for every device or (B, S); `failure_mode` scalar
    or (B,). `zimt_ion_currents`: each species' last region's ion current alone, as ZimT 5.36
    has it with several regions. `oc` (B×S or S, true at the open circuit, `V` unread there):
    where any step of the batch has it or any device a series resistance, the internal voltage
    is an unknown of every step (`newton_step_vint`), from the last one at the open circuit
    (extrapolated as the state) or the external voltage less the last current's drop, the steady
    start at 0 V where the first step is at the open circuit (transient.py:290-300, 389-405).
    `conv_var`, `tol_pois`, `tol_dens`, `tol_curr` (scalars or B): how ZimT's automatic stop
    compares two states (`TVG`'s `convVar`, `tolPois`, `tolDens`, `tolCurr`).
    `layers` (each device's `(i0, i1)`): also ZimT's tJFile columns of every step (`columns`,
    as `out["columns"][name]`, B×S or B×S×layers).
    Returns a dict: `J`, `J_ext`, `V_int`, `converged`, `iterations`, `accepted` (B×S), `stop`
    (B: 0, `STOP_STATIC` or `STOP_FAILED`), and the final state (`y` B×NP×5, `logs`, `f_bulk`, `f_interface`)."""
    d = batch
    nb = d["Vt"].shape[0]
    S = np.shape(t)[-1]
    t, V, G_frac = (np.broadcast_to(np.asarray(a, dtype=float), (nb, S)) for a in (t, V, G_frac))
    oc = np.zeros((nb, S), bool) if oc is None else np.broadcast_to(np.asarray(oc, bool), (nb, S))
    V = np.where(oc, 0.0, V)
    vint = bool(oc.any() or np.any(d["R_series"] > 0))
    track = np.zeros((nb, S), int) if track is None else np.broadcast_to(np.asarray(track), (nb, S))
    fm = np.broadcast_to(np.asarray(failure_mode), (nb,))
    check_scope(d, oc=oc, track=track, conv_var=conv_var)
    tol_pois, tol_dens, tol_curr = (np.broadcast_to(np.asarray(v, dtype=float), (nb,))
                                    for v in (tol_pois, tol_dens, tol_curr))
    conv_var = np.broadcast_to(np.asarray(conv_var), (nb,))
    by_current = bool(np.any(conv_var != 1))
    bern = dd.BERNOULLI[bernoulli_name]
    Vt = d["Vt"]
    NP = d["x"].shape[1] - 2
    ion = d["ion"]
    s = d["s"]

    # the steady state at the first step (transient.py:301-320): `_start`, then Newton
    d0 = dict(d, g_frac=G_frac[:, 0])
    V0 = np.where(oc[:, 0], 0.0, V[:, 0])
    y3, logs, _ = dd.start(d0, V0, bern, tol, max_iter)
    y3s, logs_s, J_s, ok_s, _ = dd.newton_loop(y3, logs, d0, V0, bern, tol, max_iter)
    y3 = np.where(ok_s[:, None, None], y3s, y3)
    logs = np.where(ok_s[:, None], logs_s, logs)
    la, lc = dd.point_logs(logs, ion)
    Vm = y3[..., 0]
    za, zc = la + Vm / _col(Vt), lc - Vm / _col(Vt)
    y = np.concatenate([y3, np.stack([np.where(s["a_mask"] > 0, za, 0.0),
                                      np.where(s["c_mask"] > 0, zc, 0.0)], -1)], -1)
    fb = np.zeros((nb, NP))
    fi = np.zeros((nb, NP + 1))
    J_ext_now = np.where(ok_s, J_s, 0.0) + d["G_shunt"] * V0
    dti_now = np.zeros(nb)
    t_last = np.zeros(nb)
    V_now, V_before = V0.copy(), V0.copy()
    y_prev, logs_prev = y.copy(), logs.copy()
    first = True
    track_curr = np.zeros(nb, int)
    stop = np.zeros(nb, int)
    # the automatic stop: the last state kept and the reference state, blank (G -1) at first
    cur = ref = None
    G_cur, G_ref = np.full(nb, -1.0), np.full(nb, -1.0)
    J_cur, J_ref, err_cur, err_ref = (np.zeros(nb) for _ in range(4))
    count = np.zeros(nb, int)
    caps = _caps(Vt)
    out = {k: np.zeros((nb, S)) for k in ("J", "J_ext", "V_int")}
    v_cap = dd.STEP_CAPS[0] * Vt
    cols = {}
    out.update(converged=np.zeros((nb, S), bool), iterations=np.zeros((nb, S), int),
               accepted=np.zeros((nb, S), bool))
    ma, mc = ion["a_slots"].sum(1), ion["c_slots"].sum(1)
    for k in range(S):
        t_k, V_k, G_k = t[:, k], V[:, k], G_frac[:, k]
        dti_k = np.where(t_k == 0, 0.0, 1.0 / np.where(t_k > t_last, t_k - t_last, 1.0))
        before = full_of(d, y, V_now, bern, dti_now)
        tr = {"dti": dti_k, "n": np.exp(before[:, 1:-1, 1]), "p": np.exp(before[:, 1:-1, 2]),
              "a": np.exp(before[:, 1:-1, 3]) * s["a_mask"],
              "c": np.exp(before[:, 1:-1, 4]) * s["c_mask"], "fb": fb, "fi": fi}
        trc = {"dti": dti_k, "n": np.exp(before[..., 1]), "p": np.exp(before[..., 2]),
               "a": np.exp(before[..., 3]) * ma, "c": np.exp(before[..., 4]) * mc,
               "V": before[..., 0], "fb": fb, "fi": fi,
               "ion_last": np.full(nb, bool(zimt_ion_currents))}
        moving = (dti_k > 0) & (dti_now > 0) & (not first)
        rt = np.where(moving, dti_now / np.where(moving, dti_k, 1.0), 0.0)
        guess = y + np.clip(_col(rt)[..., None] * (y - y_prev), -caps, caps)
        logs_guess = logs + np.clip(_col(rt) * (logs - logs_prev), -ION_LOG_CAP, ION_LOG_CAP)
        if vint:  # the internal voltage's start (transient.py:398-401)
            V_g = np.where(oc[:, k], V_now + np.clip(rt * (V_now - V_before), -v_cap, v_cap),
                           V_k - d["R_series"] * J_ext_now)
        else:
            V_g = V_k
        steady = dd.ion_logs(full_of(d, guess, V_g)[..., 0], ion, Vt)
        logs_guess = np.where(_col(dti_k) > 0, np.where(_col(moving), logs_guess, 0.0), steady)
        dk = dict(d, g_frac=G_k)
        if vint:
            y_new, logs_new, J, ok, it, V_new = newton_loop(
                guess, logs_guess, dk, V_g, tr, trc, bern, tol, max_iter, zimt_current,
                vint=(oc[:, k], V_k))
        else:
            y_new, logs_new, J, ok, it = newton_loop(guess, logs_guess, dk, V_k, tr, trc, bern,
                                                     tol, max_iter, zimt_current)
            V_new = V_k
        J_ext = J + d["G_shunt"] * V_new
        after = full_of(d, y_new, V_new)
        n_a, p_a = np.exp(after[..., 1]), np.exp(after[..., 2])
        fb_new = bulk_occupation(n_a[:, 1:-1], p_a[:, 1:-1], s, fb, _col(dti_k))
        fi_new = iface_occupation(n_a, p_a, d["ti"], fi, _col(dti_k))
        # ZimT's main loop (transient.py:419-445)
        running = stop == 0
        finite = np.all(np.isfinite(y_new), axis=(1, 2)) & np.all(np.isfinite(logs_new), 1)
        failed = running & ~ok & ((fm == 0) | ((fm == 2) & (track_curr == 1)))
        keep = running & ~failed & finite & (ok | (fm == 1) | ((fm == 2) & (dti_k == 0)))
        kk = keep[:, None, None]
        y, y_prev = np.where(kk, y_new, y), np.where(kk, y, y_prev)
        logs, logs_prev = (np.where(keep[:, None], logs_new, logs),
                           np.where(keep[:, None], logs, logs_prev))
        V_before, V_now = np.where(keep, V_now, V_before), np.where(keep, V_new, V_now)
        J_ext_now = np.where(keep, J_ext, J_ext_now)
        dti_now = np.where(keep, dti_k, dti_now)
        fb = np.where(keep[:, None], fb_new, fb)
        fi = np.where(keep[:, None], fi_new, fi)
        track_curr = np.where(keep, track[:, k], track_curr)
        t_last = np.where(keep, t_k, t_last)
        # ZimT's automatic stop by the last state kept (transient.py:429-442): Track 1 makes it
        # the reference where the step converged; 2 and 3 count equal states in a row (where the
        # step converged or failureMode is 1), 3 then makes it the reference
        now = summary(d, full_of(d, y_new, V_new, bern, dti_k))
        cur = now if cur is None else {f: np.where(keep[:, None], now[f], cur[f]) for f in now}
        G_cur = np.where(keep, G_k, G_cur)
        if by_current:  # the step's current and its errJ (`columns`)
            parts, _ = current_parts(dk, full_of(d, y_new, V_new, bern, dti_k), trc, bern,
                                     zimt_current)
            total = sum(parts.values())
            dev = np.concatenate([total, total[:, -1:]], 1) - _col(J)
            err = np.sqrt(np.sum(dev ** 2, 1) / (NP + 1))
            J_cur, err_cur = np.where(keep, J, J_cur), np.where(keep, err, err_cur)
        ref = {f: np.zeros_like(v) for f, v in cur.items()} if ref is None else ref
        counted = running & ~failed & ((track_curr == 2) | (track_curr == 3)) & (ok | (fm == 1))
        equal = states_equal(ref, cur, G_ref, G_cur, tol_pois, tol_dens, conv_var, tol_curr,
                             J_ref, J_cur, err_ref, err_cur)
        count = np.where(counted, np.where(equal, count + 1, 0), count)
        becomes_ref = running & ~failed & (((track_curr == 1) & ok)
                                           | ((track_curr == 3) & (ok | (fm == 1))))
        ref = {f: np.where(becomes_ref[:, None], cur[f], ref[f]) for f in cur}
        G_ref = np.where(becomes_ref, G_cur, G_ref)
        J_ref, err_ref = np.where(becomes_ref, J_cur, J_ref), np.where(becomes_ref, err_cur, err_ref)
        static = running & (count >= MIN_COUNT_STATIC)
        stop = np.where(failed, STOP_FAILED, np.where(static, STOP_STATIC, stop))
        first = False
        out["J"][:, k], out["J_ext"][:, k], out["V_int"][:, k] = J, J_ext, V_new
        if layers is not None:
            fl = full_of(d, y_new, V_new, bern, dti_k)
            parts, points = current_parts(dk, fl, trc, bern, zimt_current)
            for name, v in columns(layers, d, parts, points, fl, J, J_ext).items():
                cols.setdefault(name, np.zeros((nb, S) + v.shape[1:]))[:, k] = v
        out["converged"][:, k], out["iterations"][:, k], out["accepted"][:, k] = ok, it, keep
    out.update(stop=stop, y=y, logs=logs, f_bulk=fb, f_interface=fi)
    if layers is not None:
        out["columns"] = cols
    return out
