"""Oracle (test infrastructure): a CPU restatement of jaxdd's small-signal impedance
(src/jaxdd/impedance.py), in FP64/complex128 NumPy; devices with free mobile ions take them as
unknowns of their own (`admittance_ions`, built on `oracle.transient`'s 5×5 rows).

Only the tests import this module. It restates, one device at a time:

* `_trap_terms`, `_beyond_steady`, `_step_transfer` (continuous response), `_trap_blocks`
  (impedance.py:66-103, 197-212): the bulk traps' occupation as a state of its own;
* `_interface_beyond`, `_interface_blocks`, `_interface_rates` (impedance.py:120-194): the
  interface traps' occupation on each edge;
* `_admittance` without ions (impedance.py:230-353): the steady Jacobian plus `iω·M` and the
  traps' blocks, one complex block-tridiagonal solve per frequency for `δy = −(J + iωM)⁻¹ ∂F/∂V`,
  and the current of a time step (`batch._current_parts` with `tr`, batch.py:316-403: each
  density's change in the integrand over control-volume widths, `_sum_widths`, batch.py:406-418,
  and the displacement current) linearised; `solve_impedance` (impedance.py:365-409).

jaxdd takes the current's derivatives with `jax.jvp`; here by complex step (`current_tr` is
written for complex inputs and is analytic in them), exact to round-off.
"""

from __future__ import annotations

import warnings

import numpy as np

from jaxdd_b200.constants import Q

from . import dd


def _step_transfer(a, lap, dt=None):
    """(δf − δf₀)/δf₀ of a level of rate `a` at `iω` = `lap` (impedance.py:107-117), in the rates
    and in the charge: continuous both −iω/(iω + a); over implicit Euler's steps of `dt` (`lap`
    then `(1 − z⁻¹)/dt`) the occupation's mean over a step and its value at the step's end."""
    if dt is None:
        h = -lap / (lap + a)
        return h, h
    x = a * dt
    E, m = np.exp(-x), -np.expm1(-x) / x
    den = 1.0 - E * (1.0 - lap * dt)
    return -m * lap * dt / den, -E * lap * dt / den


def trap_terms(rec, n, p):
    """`_trap_terms` for one neutral level (Boltzmann): the rate `a`, the drive of the
    occupation in (ln n, ln p) and its part in each carrier's rate (impedance.py:66-89)."""
    Nt, Cn, Cp, nt0, pt0 = rec["Nt"], rec["Cn"], rec["Cp"], rec["nt0"], rec["pt0"]
    traps = Nt > 0
    a = Cn * (n + nt0) + Cp * (p + pt0)
    b = Cn * n + Cp * pt0
    a = np.where(traps, a, 1.0)
    f = b / a
    drive = np.stack([Cn * n * (1.0 - f), -f * Cp * p], -1)
    dR = np.where(traps, np.stack([-Nt * Cn * (n + nt0), Nt * Cp * (p + pt0)], 0), 0.0)
    return a, drive, dR


def trap_blocks(s, rec, n, p, lap, dt=None):
    """`_trap_blocks` (impedance.py:197-212): the bulk traps' correction to each interior
    point's own block (NP × 3 × 3), the continuity rows' `−fac·sC·dR·δf` (neutral levels: the
    rates only)."""
    a, drive, dR = trap_terms(rec, n, p)
    rate = drive / a[:, None] * _step_transfer(a, lap, dt)[0][:, None]
    blk = np.zeros((n.shape[0], 3, 3), complex)
    for row, k in ((1, 0), (2, 1)):
        for col in (1, 2):
            blk[:, row, col] = -(s["fac"] * s["sC"]) * dR[k] * rate[:, col - 1]
    return blk


def interface_beyond(ti, n, p, lap, dt=None):
    """`_interface_beyond` (impedance.py:120-158), one level: per edge the occupation beyond its
    steady response per unit of (ln n_L, ln n_R, ln p_L, ln p_R), in the rates and in the charge
    (`rate`, `charge`: equal but for `dt`), and its part in the four point rates and the
    charge."""
    Nt, Cn, Cp, iw = ti["Nt"], ti["Cn"], ti["Cp"], ti["iw"]
    nL, nR, pL, pR = n[:-1], n[1:], p[:-1], p[1:]
    nt0, pt0 = ti["nt0_lo"] + ti["nt0_hi"], ti["pt0_lo"] + ti["pt0_hi"]
    traps = Nt > 0
    a = Cn * (nL + nR + nt0) + Cp * (pL + pR + pt0)
    b = Cn * (nL + nR) + Cp * pt0
    an, bp = Cn * Nt, Cp * Nt
    dR = np.stack([-iw * an * (nL + ti["nt0_lo"]), -iw * an * (nR + ti["nt0_hi"]),
                   iw * bp * (pL + ti["pt0_lo"]), iw * bp * (pR + ti["pt0_hi"]),
                   -ti["charge"] * 0.5 * Nt * iw])
    fa = b / np.where(a > 0, a, 1.0)
    # d a and d b in each logarithm: n_L, n_R (C_n n), p_L, p_R (C_p p; b has none)
    da = np.stack([Cn * nL, Cn * nR, Cp * pL, Cp * pR], -1)
    db = np.stack([Cn * nL, Cn * nR, 0 * pL, 0 * pR], -1)
    drive = db - fa[:, None] * da
    a = np.where(traps, a, 1.0)
    unit = drive / a[:, None]
    h_rate, h_charge = _step_transfer(a, lap, dt)
    return unit * h_rate[:, None], unit * h_charge[:, None], np.where(traps, dR, 0.0)


def interface_blocks(s, ti, n, p, lap, dt=None):
    """`_interface_blocks` (impedance.py:161-194): each edge's occupation beyond its steady
    response in its two points' rates and charge, as corrections to (A, B, C)."""
    rate, charge, dR = interface_beyond(ti, n, p, lap, dt)
    NP = n.shape[0] - 2

    def block(side, cols):
        jn, jp = (0, 2) if cols == 0 else (1, 3)
        rows = [(dR[4], charge), (dR[0 if side == 0 else 1], rate),
                (dR[2 if side == 0 else 3], rate)]
        return np.stack([np.stack([d * r[:, jn], d * r[:, jp]], -1) for d, r in rows], -2)

    def scaled(b, k):
        rs = np.stack([Q * s["sP"][k], -s["fac"][k] * s["sC"][k], -s["fac"][k] * s["sC"][k]], -1)
        return np.concatenate([np.zeros_like(b[..., :1]), b], -1) * rs[..., None]

    e = np.arange(1, NP)
    dA = np.zeros((NP, 3, 3), complex)
    dB = np.zeros((NP, 3, 3), complex)
    dC = np.zeros((NP, 3, 3), complex)
    dB[e - 1] += scaled(block(0, 0)[e], e - 1)
    dB[e] += scaled(block(1, 1)[e], e)
    dC[e - 1] += scaled(block(0, 1)[e], e - 1)
    dA[e] += scaled(block(1, 0)[e], e)
    return dA, dB, dC


def interface_rates(ti, n, p, lap, dy3, dt=None):
    """`_interface_rates` (impedance.py:178-194 region): each point's electron and hole rate of
    the interface traps beyond their steady occupation at the response `dy3`."""
    rate, _, dR = interface_beyond(ti, n, p, lap, dt)
    full = np.pad(dy3, ((1, 1), (0, 0)))
    logs = np.stack([full[:-1, 1], full[1:, 1], full[:-1, 2], full[1:, 2]], -1)
    df = np.sum(rate * logs, -1)

    def points(lo, hi):
        return np.concatenate([lo[:1], hi[:-1] + lo[1:], hi[-1:]])

    return points(dR[0] * df, dR[1] * df), points(dR[2] * df, dR[3] * df)


def current_tr(d, full, dti, before, Vbefore, width, dU=None, dRi=None, simss=False):
    """`batch._current` over a time step (`tr`: the state `before`, `dti`, control-volume widths;
    no ions, no bulk occupations carried; `dU`, `dRi` each carrier's rates beyond the steady
    traps'): one lane of the oracle's tree `d` (1-lane arrays), `full` (NP + 2) × 3, complex
    allowed (complex-step derivatives). Where `curr_diff` each interval carries its
    Scharfetter–Gummel flux (`Calc_Curr_Diff`, batch.py:383-386) with SIMsalabim's Bernoulli
    function if `simss`."""
    V, n, p = full[:, 0], np.exp(full[:, 1]), np.exp(full[:, 2])
    Vt, x, h, L = d["Vt"][0], d["x"][0], d["h"][0], d["L"][0]
    NP = x.shape[0] - 2
    rec = {k: v[0] for k, v in d["rec"].items()}
    ti = {k: v[0] for k, v in d["ti"].items()}
    g_frac = d["g_frac"][0]
    R, _, _ = dd._recombination(n[None], p[None], {k: v[None] for k, v in rec.items()})
    R = R[0]
    if np.any(ti["Nt"] > 0):
        val, _ = dd._iface_edges(n[:-1][None], n[1:][None], p[:-1][None], p[1:][None],
                                 {k: v[None] for k, v in ti.items()})
        val = val[:, 0]

        def points(lo, hi):
            return np.concatenate([lo[:1], hi[:-1] + lo[1:], hi[-1:]])

        Rin, Rip = points(val[0], val[1]), points(val[2], val[3])
    else:
        Rin = Rip = np.zeros_like(R)
    if dRi is not None:
        Rin, Rip = Rin + dRi[0], Rip + dRi[1]
    dx = np.diff(x[:NP + 1])
    G = d["G"][0]

    def carrier(sn, Vg, dens, mu, R_i, bef, dU_c):
        U = R + R_i - G * g_frac + (0.0 if dU_c is None else dU_c)
        U = U.astype(complex)
        U[0] = 0.0
        U[-1] = 0.0
        change = dti * (dens - bef)
        change = change.astype(complex)
        change[0] = 0.0
        U = U + change
        ev = np.exp(sn * Vg[:NP + 1] / Vt)
        int_u = np.concatenate([[0.0], np.cumsum(0.5 * dx * (U[:NP] + U[1:NP + 1]))])
        single = np.sum(0.5 * dx * (ev[:-1] / mu[:NP] + ev[1:] / mu[1:NP + 1]))
        double = np.sum(0.5 * dx * (ev[:-1] * int_u[:-1] / mu[:NP]
                                    + ev[1:] * int_u[1:] / mu[1:NP + 1]))
        K = (Vt * (sn * dens[NP + 1] * np.exp(sn * Vg[NP + 1] / Vt)
                   - sn * dens[0] * np.exp(sn * Vg[0] / Vt)) - sn * double) / single
        J = Q * K + np.concatenate([[0.0], np.cumsum(sn * Q * L * width[1:NP + 1] * U[1:NP + 1])])
        if d["curr_diff"][0] > 0:
            dVg = sn * np.diff(Vg) / Vt
            J = sn * Q * mu[:NP + 1] * Vt * (dens[1:] * dd.bern_complex(-dVg, simss)
                                             - dens[:-1] * dd.bern_complex(dVg, simss)) / (L * h[:NP + 1])
        through = sn * 0.5 * Q * L * h[:NP + 1] * (R_i[:NP + 1] + R_i[1:])
        return np.where(d["iface"][0], np.roll(J, 1) + through, J)

    sign = -d["left_elec"][0]
    dUn, dUp = (None, None) if dU is None else dU
    Jn = sign * carrier(-1.0, V + d["offset_n"][0], n, d["mu_n"][0], Rin, before[0], dUn)
    Jp = sign * carrier(1.0, V + d["offset_p"][0], p, d["mu_p"][0], Rip, before[1], dUp)
    JD = sign * d["eps"][0][:NP + 1] * (np.diff(V) - np.diff(Vbefore)) * dti / (L * h[:NP + 1])
    hh = h[:NP + 1]
    return np.sum(hh * (Jn + Jp + JD)) / np.sum(hh)


def admittance(d, full0, Vint, laps, bern, dt=None):
    """One device's δJ/δV_int at each `iω` of `laps` about its steady state `full0`
    (`_admittance` without ions, impedance.py:230-353). `d` the oracle's 1-lane tree."""
    s = {k: v[0] for k, v in d["s"].items()}
    rec = {k: v[0] for k, v in d["rec"].items()}
    ti = {k: v[0] for k, v in d["ti"].items()}
    y3 = full0[1:-1]
    NP = y3.shape[0]
    n, p = np.exp(y3[:, 1]), np.exp(y3[:, 2])
    n_full, p_full = np.exp(full0[:, 1]), np.exp(full0[:, 2])
    zero = np.zeros((1, NP))
    F, A, Bb, C, _ = dd.assemble(full0[None], d["s"], d["ti"], d["Vt"], d["g_frac"], zero, zero,
                                 bern)
    A, Bb, C = A[0], Bb[0], C[0]
    M = np.stack([np.zeros(NP), -s["fac"] * n * s["sC"], -s["fac"] * p * s["sC"]], -1)
    # the drive: the residual's derivative in V_int, through the contacts (batch._bounds)
    e = d["left_elec"][0]
    dF = np.zeros((NP, 3))
    dF[0] += A[0][:, 0] * 0.5 * e
    dF[-1] += C[-1][:, 0] * (-0.5 * e)
    hh = d["h"][0][:NP + 1]
    width = np.concatenate([hh[:1], 0.5 * (hh[:-1] + hh[1:])])
    before = (n_full, p_full)
    Vb = full0[:, 0]
    def full_of(y, V):  # batch._bounds at a (complex) voltage
        left = [d["V0"][0] + 0.5 * e * V, d["ln_n_left"][0], d["ln_p_left"][0]]
        right = [d["VL"][0] - 0.5 * e * V, d["ln_n_right"][0], d["ln_p_right"][0]]
        return np.concatenate([np.array([left], complex), y, np.array([right], complex)], 0)

    h_cs = 1e-30

    simss = bern is dd.bern_simss

    def linear(dy_real, dV, dti):  # J_y dy + J_V dV at dti, by complex step
        y = y3 + 1j * h_cs * dy_real
        V = Vint + 1j * h_cs * dV
        return np.imag(current_tr(d, full_of(y, V), dti, before, Vb, width,
                                  simss=simss)) / h_cs

    def rates(dU, dRi):  # linear in both
        J0 = current_tr(d, full0.astype(complex), 0.0, before, Vb, width, simss=simss)
        J1 = current_tr(d, full0.astype(complex), 0.0, before, Vb, width, dU, dRi, simss=simss)
        return J1 - J0

    out = []
    for lap in laps:
        Bl = Bb + lap * M[:, :, None] * np.eye(3)[None]
        Bl = Bl + trap_blocks(s, {k: v[1:-1] for k, v in rec.items()}, n, p, lap, dt)
        Al, Cl = A.astype(complex), C.astype(complex)
        if np.any(ti["Nt"] > 0):
            dA, dB, dC = interface_blocks(s, ti, n_full, p_full, lap, dt)
            Al, Bl, Cl = Al + dA, Bl + dB, Cl + dC
        rhs = (-dF).astype(complex)[:, :, None]
        dy = dd.block_thomas(Al[None], Bl[None], Cl[None], rhs[None])[0, :, :, 0]
        J0 = linear(dy.real, 1.0, 0.0) + 1j * linear(dy.imag, 0.0, 0.0)
        J1 = linear(dy.real, 1.0, 1.0) + 1j * linear(dy.imag, 0.0, 1.0)
        # the bulk traps' rates beyond their steady occupation (`beyond`)
        a, drive, dR = trap_terms({k: v[1:-1] for k, v in rec.items()}, n, p)
        rate = drive / a[:, None] * _step_transfer(a, lap, dt)[0][:, None]
        df = rate[:, 0] * dy[:, 1] + rate[:, 1] * dy[:, 2]
        pad = np.zeros(1)
        dUn = np.concatenate([pad, dR[0] * df, pad])
        dUp = np.concatenate([pad, dR[1] * df, pad])
        if np.any(ti["Nt"] > 0):
            dRn, dRp = interface_rates(ti, n_full, p_full, lap, dy, dt)
        else:
            dRn = dRp = np.zeros(NP + 2, complex)
        Ju = rates((dUn, dUp), (dRn, dRp))
        out.append(J0 + lap * (J1 - J0) + Ju)
    return np.array(out)


def admittance_ions(d, full0, Vint, laps, bern, dt=None):
    """One device's δJ/δV_int at each `iω` of `laps` with its mobile ions as unknowns of their
    own (`_admittance` with `ions`, impedance.py:242-353): the 5×5 blocks of a time step of
    `dti` = 1 from the steady state `full0` ((NP + 2) × 5: V, ln n, ln p, ln a, ln c; the
    ions' 0 outside their regions) with the traps steady (`oracle.transient.assemble`),
    `Bb + (iω − 1)·M` on the diagonal, the traps' blocks on the carriers' 3×3, the ion slots as
    a border keeping each region's number (`_ion_constraints_time`), and the current of a time
    step linearised (the ions' currents included) by complex step."""
    from . import transient
    s = {k: v[0] for k, v in d["s"].items()}
    rec = {k: v[0] for k, v in d["rec"].items()}
    ti = {k: v[0] for k, v in d["ti"].items()}
    ion = d["ion"]
    y = full0[1:-1]
    NP = y.shape[0]
    K = ion["a_slots"].shape[1] + ion["c_slots"].shape[1]
    logs = np.zeros((1, K))
    n, p = np.exp(y[:, 1]), np.exp(y[:, 2])
    n_full, p_full = np.exp(full0[:, 1]), np.exp(full0[:, 2])
    am, cm = s["a_mask"], s["c_mask"]
    tr = {"dti": np.array([1.0]), "n": n[None], "p": p[None], "a": (np.exp(y[:, 3]) * am)[None],
          "c": (np.exp(y[:, 4]) * cm)[None], "fb": None, "fi": None}
    _, A, Bb, C, U, M = transient.assemble(full0[None], d, tr, logs, bern, steady_traps=True,
                                           mass=True)
    A, Bb, C, U, M = A[0], Bb[0], C[0], U[0], M[0]
    # each slot's number, the contacts' ions from their neighbours where a region reaches one
    # (`_ion_full` at the step's dti = 1): its derivatives in the interior unknowns, W, and in
    # V_int (through the contacts' potentials), dg, by complex step
    full1, dVc = transient.ion_full(d, full0[None], bern, np.array([1.0]))
    _, W, D = transient.constraints(full1, logs, ion, dVc)
    W, D = W[0], D[0]
    g_of = transient.full_of(d, y[None].astype(complex), np.array([Vint + 1j * 1e-30]), bern,
                             np.array([1.0]))
    with warnings.catch_warnings():  # W of a complex state, unused, cast to real
        warnings.simplefilter("ignore", np.exceptions.ComplexWarning)
        dg = np.imag(transient.constraints(g_of, logs, ion)[0][0]) / 1e-30
    e = d["left_elec"][0]
    dF = np.zeros((NP, 5))
    dF[0] += A[0][:, 0] * 0.5 * e
    dF[-1] += C[-1][:, 0] * (-0.5 * e)
    ma, mc = ion["a_slots"][0].sum(0), ion["c_slots"][0].sum(0)
    tr0 = {"dti": np.array([0.0]), "n": n_full[None], "p": p_full[None],
           "a": (np.exp(full0[:, 3]) * ma)[None], "c": (np.exp(full0[:, 4]) * mc)[None],
           "V": full0[None, :, 0]}
    h_cs = 1e-30

    def total(y_, V_, dti, dU=None, dRi=None):  # the contacts' ions `_ion_full`'s at dti
        t = dict(tr0, dti=np.array([dti]))
        full = transient.full_of(d, y_[None], np.array([V_]), bern, np.array([dti]))
        return transient.current(d, full, t, bern, False, steady_traps=True, dU=dU, dRi=dRi)[0]

    def linear(dy_real, dV, dti):  # J_y dy + J_V dV at dti, by complex step
        return np.imag(total(y + 1j * h_cs * dy_real, Vint + 1j * h_cs * dV, dti)) / h_cs

    def rates(dU, dRi):
        J0 = total(y.astype(complex), complex(Vint), 0.0)
        J1 = total(y.astype(complex), complex(Vint), 0.0, tuple(v[None] for v in dU),
                   tuple(v[None] for v in dRi))
        return J1 - J0

    eye = np.eye(5)
    out = []
    for lap in laps:
        Bl = Bb + ((lap - 1.0) * M)[:, :, None] * eye[None]
        Bl[:, :3, :3] += trap_blocks(s, {k: v[1:-1] for k, v in rec.items()}, n, p, lap, dt)
        Al, Cl = A.astype(complex), C.astype(complex)
        if np.any(ti["Nt"] > 0):
            dA, dB, dC = interface_blocks(s, ti, n_full, p_full, lap, dt)
            Al[:, :3, :3] += dA
            Bl[:, :3, :3] += dB
            Cl[:, :3, :3] += dC
        rhs = np.concatenate([(-dF).astype(complex)[:, :, None], U.astype(complex)], -1)
        X = transient.block_thomas(Al[None], Bl[None], Cl[None], rhs[None])[0]
        XF, XU = X[..., 0], X[..., 1:]
        schur = D - np.einsum("kir,irl->kl", W, XU)
        z = np.linalg.solve(schur, -dg - np.einsum("kir,ir->k", W, XF))
        dy = XF - XU @ z
        J0 = linear(dy.real, 1.0, 0.0) + 1j * linear(dy.imag, 0.0, 0.0)
        J1 = linear(dy.real, 1.0, 1.0) + 1j * linear(dy.imag, 0.0, 1.0)
        a, drive, dR = trap_terms({k: v[1:-1] for k, v in rec.items()}, n, p)
        rate = drive / a[:, None] * _step_transfer(a, lap, dt)[0][:, None]
        df = rate[:, 0] * dy[:, 1] + rate[:, 1] * dy[:, 2]
        pad = np.zeros(1)
        dUn = np.concatenate([pad, dR[0] * df, pad])
        dUp = np.concatenate([pad, dR[1] * df, pad])
        if np.any(ti["Nt"] > 0):
            dRn, dRp = interface_rates(ti, n_full, p_full, lap, dy[:, :3], dt)
        else:
            dRn = dRp = np.zeros(NP + 2, complex)
        Ju = rates((dUn, dUp), (dRn, dRp))
        out.append(J0 + lap * (J1 - J0) + Ju)
    return np.array(out)


def solve_impedance(devices, frequencies, voltage=0.0, tol=1e-10, max_iter=60,
                    bernoulli_name="exact", dt=None):
    """`solve_impedance` (impedance.py:365-409): `(Y, Z, J, converged)`, Y and Z devices ×
    frequencies. Devices with free mobile ions take them as unknowns of their own
    (`admittance_ions`); ions frozen at a pre-bias are refused, as the reference refuses them."""
    frequencies = np.atleast_1d(np.asarray(frequencies, dtype=float))
    laps = 1j * 2 * np.pi * frequencies
    if dt is not None:  # implicit Euler's steps of dt: iω as (1 − z⁻¹)/dt (impedance.py:379-383)
        laps = -np.expm1(-laps * dt) / dt
    bern = dd.BERNOULLI[bernoulli_name]
    Y, J, ok = [], [], []
    for dev in devices:
        d = dd.prepare([dev])
        ions = np.any(d["ion"]["a_totals"] > 0) or np.any(d["ion"]["c_totals"] > 0)
        if ions and dev.pre_cond and dev.fix_ions:
            raise NotImplementedError("impedance with ions frozen at a pre-bias")
        st = dd.solve_states(d, [float(voltage)], tol=tol, max_iter=max_iter,
                             bernoulli_name=bernoulli_name)
        full0 = np.stack([st["V"][0, 0], np.log(st["n"][0, 0]), np.log(st["p"][0, 0])], -1)
        if ions:
            a_m = np.asarray(dev.anion_mask, bool)
            c_m = np.asarray(dev.cation_mask, bool)
            la = np.where(a_m, np.log(np.where(a_m, st["anion"][0, 0], 1.0)), 0.0)
            lc = np.where(c_m, np.log(np.where(c_m, st["cation"][0, 0], 1.0)), 0.0)
            full5 = np.concatenate([full0, la[:, None], lc[:, None]], -1)
            full5[0, 3:] = 0.0
            full5[-1, 3:] = 0.0
            Y.append(admittance_ions(d, full5, float(voltage), laps, bern, dt))
        else:
            Y.append(admittance(d, full0, float(voltage), laps, bern, dt))
        J.append(st["J"][0, 0])
        ok.append(st["converged"][0, 0])
    Y = np.array(Y)
    G_shunt = np.array([1.0 / d.R_shunt if d.R_shunt > 0 else 0.0 for d in devices])
    R_series = np.array([d.R_series for d in devices])
    Z = 1.0 / (Y + G_shunt[:, None]) + R_series[:, None]
    return Y, Z, np.array(J), np.array(ok)
