// Device code shared by the transient (dd_transient.cu) and the impedance with mobile ions
// (dd_impedance.cu): a point of the 5-unknown state (V, ln n, ln p, ln a, ln c), the traps'
// occupation over a time step (`_trap_step`, solver.py:594-614), the ions' Scharfetter-Gummel
// fluxes, one row's residual and 5x5 blocks over a step (`_assemble_ions`, solver.py:1364-1475),
// and the 5x5 block solve by its partition (`_inverse5`, solver.py:1505-1517). Inline: each
// translation unit gets its own copy.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "dd_layout.h"
#include "dd_physics.cuh"
#include "../../include/jaxdd_b200.h"

namespace dd {
namespace tr {

enum TField { T_EPS = 0, T_MUA, T_MUC };


// A point of the 5-unknown state and what the rows need of it.
struct TP {
  Pt c;           // V, ln n, ln p, n, p, offsets, slots (dd_physics.cuh)
  double la, lc;  // ln a, ln c (0 outside their regions)
  double a, c2;   // exp(la), exp(lc)
};

struct View {
  Lane L;
  const double* X;
  double* Yb;
  size_t ybuf;
  int simss, zimt;
  int ion_last = 0;  // each species' last ion region's current alone (ZimT 5.36's)
  const double* BD;  // the step's state before it as densities [np+2][4][Bp] (n, p, a, c), or null
  __device__ __forceinline__ double x(int k, int f) const {
    return __ldg(X + ((size_t)k * DD_NT + f) * L.Bp + L.l);
  }
  __device__ __forceinline__ double* y(int buf, int k, int c) const {
    return Yb + buf * ybuf + ((size_t)k * 5 + c) * L.Bp + L.l;
  }
};

// A point of buffer `buf` (interior) or a contact at internal voltage `Vint`.
__device__ __forceinline__ void load_point(const View& W, int buf, int k, double Vint, TP& P) {
  const Lane& L = W.L;
  if (k == 0 || k == L.NP + 1) {
    contact(L, k != 0, Vint, P.c);
    P.la = 0.0; P.lc = 0.0;
  } else {
    P.c.V = *W.y(buf, k, 0); P.c.lnn = *W.y(buf, k, 1); P.c.lnp = *W.y(buf, k, 2);
    P.la = *W.y(buf, k, 3); P.lc = *W.y(buf, k, 4);
  }
  P.c.n = exp(P.c.lnn);
  P.c.p = exp(P.c.lnp);
  P.c.offn = L.st(k, S_OFFN);
  P.c.offp = L.st(k, S_OFFP);
  P.c.sl = slots_at(L, k);
  // the ions' densities where they are mobile (elsewhere their unknown is held at 0)
  P.a = P.c.sl.a >= 0 ? exp(P.la) : 1.0;
  P.c2 = P.c.sl.c >= 0 ? exp(P.lc) : 1.0;
  P.c.da = P.c.sl.a >= 0 ? P.a : 0.0;
  P.c.dc = P.c.sl.c >= 0 ? P.c2 : 0.0;
}

// A contact's ions where a region reaches it (`_ion_full`, solver.py:1315-1346): from its
// neighbour in buffer `buf`, so that nothing flows over the contact's interval,
// ln a_0 = ln a_1 + ln(B(x)/B(-x)) with x = (V_1 - V_0)/V_T (the cations' the other way, the right
// contact's mirrored), Boltzmann's (the ratio -x) in the steady state dti = 0. `dr`, if given:
// d ln a / d V of the neighbour (the cations' its negative). `nbp`, if given: the neighbour's
// point itself (a state along a tangent) instead of buffer `buf`'s. A no-op on interior points
// and where no region reaches the contact.
__device__ __forceinline__ void contact_ions(const View& W, int buf, int k, double dti, TP& P,
                                             double* dr = nullptr, const TP* nbp = nullptr) {
  const Lane& L = W.L;
  if ((k != 0 && k != L.NP + 1) || (P.c.sl.a < 0 && P.c.sl.c < 0)) return;
  const bool right = k != 0;
  const int nb = right ? L.NP : 1;
  const double Vn = nbp ? nbp->c.V : *W.y(buf, nb, 0);
  const double x = (right ? P.c.V - Vn : Vn - P.c.V) * L.iVt;
  double r = -x, drx = -1.0;
  if (dti > 0.0) {
    double Bf, Bb, dBf, dBb;
    bern_pair(x, W.simss, Bf, Bb, dBf, dBb);
    r = log(Bf) - log(Bb);
    drx = dBf / Bf + dBb / Bb;
  }
  const double s = right ? -1.0 : 1.0;  // the step from the neighbour, anions
  if (dr) *dr = drx * L.iVt;  // on either side r'(x) / V_T
  if (P.c.sl.a >= 0) {
    P.la = (nbp ? nbp->la : *W.y(buf, nb, 3)) + s * r;
    P.a = exp(P.la);
    P.c.da = P.a;
  }
  if (P.c.sl.c >= 0) {
    P.lc = (nbp ? nbp->lc : *W.y(buf, nb, 4)) - s * r;
    P.c2 = exp(P.lc);
    P.c.dc = P.c2;
  }
}

// ------------------------------------------------------------------------------------ traps

// A level's occupation over a step of 1/dti from f_old (`_trap_step` with `empty`): its mean,
// its value at the step's end and the mean of the empty share, with their derivatives in n and
// in p (not in their logarithms). dti = 0: the steady occupation.
struct TrapStep {
  double mean, end, vac;
  double mn, en, vn, mp, ep, vp;
  double mf, Ef;  // d mean / d f_old (= -d vac / d f_old) and d end / d f_old
};

__device__ __forceinline__ void trap_step(double Cn, double Cp, double nt0, double pt0, double n,
                                          double p, double f_old, double dti, TrapStep& o) {
  double a = Cn * (n + nt0) + Cp * (p + pt0);
  const bool pos = a > 0.0;
  if (!pos) a = 1.0;
  const double ia = 1.0 / a;
  const double da_n = pos ? Cn : 0.0, da_p = pos ? Cp : 0.0;
  const double steady = (Cn * n + Cp * pt0) * ia, vac_s = (Cn * nt0 + Cp * p) * ia;
  const double ds_n = (Cn - steady * da_n) * ia, ds_p = -steady * da_p * ia;
  const double dv_n = -vac_s * da_n * ia, dv_p = (Cp - vac_s * da_p) * ia;
  double E = 0.0, m = 0.0, dm = 0.0, dx_n = 0.0, dx_p = 0.0;
  if (dti > 0.0) {
    const double idti = 1.0 / dti;
    const double x = a * idti, ix = dti * ia;
    E = exp(-x);
    m = -expm1(-x) * ix;
    dm = (E - m) * ix;
    dx_n = da_n * idti;
    dx_p = da_p * idti;
  }
  const double gap = f_old - steady, vgap = (1.0 - f_old) - vac_s;
  o.mean = steady + gap * m;
  o.end = steady + gap * E;
  o.vac = vac_s + vgap * m;
  o.mn = ds_n * (1.0 - m) + gap * dm * dx_n;
  o.en = ds_n * (1.0 - E) - gap * E * dx_n;
  o.vn = dv_n * (1.0 - m) + vgap * dm * dx_n;
  o.mp = ds_p * (1.0 - m) + gap * dm * dx_p;
  o.ep = ds_p * (1.0 - E) - gap * E * dx_p;
  o.vp = dv_p * (1.0 - m) + vgap * dm * dx_p;
  o.mf = m;
  o.Ef = E;
}

// Each carrier's recombination over the step at point k (`_bulk_rates` with the traps'
// occupation `fb`, solver.py:680-700) and their derivatives in ln n, ln p.
__device__ __forceinline__ void bulk_rates(const Lane& L, int k, double n, double p, double fb,
                                           double dti, double& Rn, double& Rp, double& dRn_n,
                                           double& dRn_p, double& dRp_n, double& dRp_p) {
  const double kd = L.st(k, S_KD), ni2 = L.st(k, S_NI2), Nt = L.st(k, S_NT);
  const double direct = kd * (n * p - ni2);
  Rn = direct; Rp = direct;
  double an = kd * p, ap = kd * n, bn = kd * p, bp = kd * n;  // d/dn, d/dp of Rn; of Rp
  if (Nt > 0.0) {
    const double Cn = L.st(k, S_CNT), Cp = L.st(k, S_CPT);
    const double nt0 = L.st(k, S_NT0), pt0 = L.st(k, S_PT0);
    TrapStep o;
    trap_step(Cn, Cp, nt0, pt0, n, p, fb, dti, o);
    Rn += Nt * Cn * (n * o.vac - nt0 * o.mean);
    Rp += Nt * Cp * (p * o.mean - pt0 * o.vac);
    an += Nt * Cn * (o.vac + n * o.vn - nt0 * o.mn);
    ap += Nt * Cn * (n * o.vp - nt0 * o.mp);
    bn += Nt * Cp * (p * o.mn - pt0 * o.vn);
    bp += Nt * Cp * (o.mean + p * o.mp - pt0 * o.vp);
  }
  dRn_n = n * an; dRn_p = p * ap;
  dRp_n = n * bn; dRp_p = p * bp;
}

__device__ __forceinline__ double bulk_end(const Lane& L, int k, double n, double p, double fb,
                                           double dti) {
  TrapStep o;
  trap_step(L.st(k, S_CNT), L.st(k, S_CPT), L.st(k, S_NT0), L.st(k, S_PT0), n, p, fb, dti, o);
  return o.end;
}

// Interface traps of one interval (table row t) over the step (`_interface_edges` with `f_old`,
// solver.py:814-850): v = (Rn_L, Rn_R, Rp_L, Rp_R, Q) and their derivatives in
// ln nL, ln nR, ln pL, ln pR; `end` the occupation at the step's end.
static __device__ void iface_edge_t(const Lane& L, int t, double nL, double nR, double pL,
                                    double pR, double f_old, double dti, Iface& o, bool derivs,
                                    double* end) {
  const double Nt = L.itab(t, I_NT), Cn = L.itab(t, I_CN), Cp = L.itab(t, I_CP);
  const double nlo = L.itab(t, I_NT0LO), nhi = L.itab(t, I_NT0HI);
  const double plo = L.itab(t, I_PT0LO), phi = L.itab(t, I_PT0HI);
  const double iw = L.itab(t, I_IW);
  const double hq = L.itab(t, I_CHARGE) * 0.5 * Nt * iw, cwe = L.itab(t, I_CWE);
  const double an = Cn * Nt, bp = Cp * Nt;
  TrapStep s;
  trap_step(Cn, Cp, nlo + nhi, plo + phi, nL + nR, pL + pR, f_old, dti, s);
  const bool traps = Nt > 0.0;
  const double full = traps ? s.mean : 0.0, fend = traps ? s.end : 0.0;
  const double empty = traps ? s.vac : 0.0;
  if (end) *end = fend;
  o.v[0] = iw * an * (nL * empty - nlo * full);
  o.v[1] = iw * an * (nR * empty - nhi * full);
  o.v[2] = iw * bp * (pL * full - plo * empty);
  o.v[3] = iw * bp * (pR * full - phi * empty);
  o.v[4] = hq * (cwe - fend);
  if (!derivs) return;
#pragma unroll
  for (int w = 0; w < 4; ++w) {
    const double dens = w == 0 ? nL : (w == 1 ? nR : (w == 2 ? pL : pR));
    double dF, dE, dEnd;
    if (w < 2) { dF = s.mn * dens; dE = s.vn * dens; dEnd = s.en * dens; }
    else { dF = s.mp * dens; dE = s.vp * dens; dEnd = s.ep * dens; }
    if (!traps) { dF = 0.0; dE = 0.0; dEnd = 0.0; }
    o.d[w][0] = iw * an * ((w == 0 ? nL * empty : 0.0) + nL * dE - nlo * dF);
    o.d[w][1] = iw * an * ((w == 1 ? nR * empty : 0.0) + nR * dE - nhi * dF);
    o.d[w][2] = iw * bp * ((w == 2 ? pL * full : 0.0) + pL * dF - plo * dE);
    o.d[w][3] = iw * bp * ((w == 3 ? pR * full : 0.0) + pR * dF - phi * dE);
    o.d[w][4] = -hq * dEnd;
  }
}

// ------------------------------------------------------------------------------------ ions

// One interval's Scharfetter-Gummel flux of a species between points a (left) and b (right) at
// mobility c/V_T, and its derivatives in x = (V_b - V_a)/V_T and in ln n_a, ln n_b: anions as
// electrons F = c (B(x) n_b - B(-x) n_a), cations as holes F = c (B(x) n_a - B(-x) n_b).
struct IonIv {
  double F, gx, da, db;
};

__device__ __forceinline__ void ion_iv(double sn, double x, double na, double nb, double c,
                                       int simss, IonIv& o) {
  double Bf, Bb, dBf, dBb;
  bern_pair(x, simss, Bf, Bb, dBf, dBb);
  if (sn < 0) {
    o.F = c * (Bf * nb - Bb * na);
    o.gx = c * (dBf * nb + dBb * na);
    o.da = -c * Bb * na;
    o.db = c * Bf * nb;
  } else {
    o.F = c * (Bf * na - Bb * nb);
    o.gx = c * (dBf * na + dBb * nb);
    o.da = c * Bf * na;
    o.db = -c * Bb * nb;
  }
}

// Both species' fluxes over interval k (points a = k, b = k + 1) where both points are in a
// region of that species (zero otherwise): what row k takes as its right interval and row k + 1
// as its left one.
__device__ __forceinline__ void ion_ivs(const View& W, int k, const TP& a, const TP& b,
                                        IonIv (&o)[2]) {
  const Lane& L = W.L;
#pragma unroll
  for (int sp = 0; sp < 2; ++sp) {
    const bool both = sp == 0 ? (a.c.sl.a >= 0 && b.c.sl.a >= 0) : (a.c.sl.c >= 0 && b.c.sl.c >= 0);
    if (!both) { o[sp] = IonIv{0.0, 0.0, 0.0, 0.0}; continue; }
    const double c = L.Vt * W.x(k, sp == 0 ? T_MUA : T_MUC);
    ion_iv(sp == 0 ? -1.0 : 1.0, (b.c.V - a.c.V) * L.iVt, sp == 0 ? a.a : a.c2,
           sp == 0 ? b.a : b.c2, c, W.simss, o[sp]);
  }
}

// ------------------------------------------------------------------------------------ rows

// Row i's residual (as -F in r), blocks A, B, C (5x5) and slot columns U (5xK) over the step
// (`_assemble_ions` with `_assemble`'s carriers' rows and their time terms). `bn`, `bpd`, `ba`,
// `bc`: the point's densities before the step; `fb` its bulk traps' occupation, `fim`, `fii`
// those of its two intervals' interface traps.
template <int K, bool STEADY = false>
__device__ __forceinline__ void row5(const View& W, int i, const TP& pm, const TP& pc,
                                     const TP& pn, const Flux& el, const Flux& er, double hm,
                                     double hp, int ifk_m, int ifk_i, double dti, double fb,
                                     double fim, double fii, double bn, double bpd, double ba,
                                     double bc, const double* logs, double (&A)[5][5],
                                     double (&B)[5][5], double (&Cm)[5][5], double (&r)[5],
                                     double (&U)[5][K], double* mass = nullptr,
                                     double* tang = nullptr, const double* elogs = nullptr,
                                     const IonIv* ivl = nullptr, const IonIv* ivr = nullptr) {
  const Lane& L = W.L;
  const double iVt = L.iVt;
  const double facl = L.st(i, S_FACL), facm = L.st(i, S_FACM), facu = L.st(i, S_FACU);
  const double fac = L.st(i, S_FAC), sP = L.st(i, S_SP), sC = L.st(i, S_SC);
#pragma unroll
  for (int a = 0; a < 5; ++a) {
#pragma unroll
    for (int b = 0; b < 5; ++b) { A[a][b] = 0.0; B[a][b] = 0.0; Cm[a][b] = 0.0; }
#pragma unroll
    for (int k = 0; k < K; ++k) U[a][k] = 0.0;
  }
  double Rn, Rp, dRn_n, dRn_p, dRp_n, dRp_p;
  if (STEADY) {  // the traps at their steady occupation (`_time_terms` without occupations)
    recomb(L, i, pc.c.n, pc.c.p, Rn, dRn_n, dRn_p);
    Rp = Rn; dRp_n = dRn_n; dRp_p = dRn_p;
  } else {
    bulk_rates(L, i, pc.c.n, pc.c.p, fb, dti, Rn, Rp, dRn_n, dRn_p, dRp_n, dRp_p);
  }
  const double gen = L.st(i, S_G) * L.gfrac;
  double elec = hm * er.Fn - hp * el.Fn + fac * (gen - Rn);
  double hole = hp * el.Fp - hm * er.Fp + fac * (gen - Rp);
  const double anion = pc.c.da, cation = pc.c.dc;
  double pois = facl * pm.c.V + facm * pc.c.V + facu * pn.c.V -
                Q * (pc.c.n - pc.c.p + L.st(i, S_DOP) + L.afix(i) + anion - L.cfix(i) - cation);
  // Poisson's row: the ions' densities are unknowns of their own, none follows V
  A[0][0] = facl * sP;
  Cm[0][0] = facu * sP;
  B[0][0] = facm * sP;
  B[0][1] = -Q * pc.c.n * sP;
  B[0][2] = Q * pc.c.p * sP;
  B[0][3] = -Q * anion * sP;
  B[0][4] = Q * cation * sP;
  A[1][0] = -hp * el.n0V * sC; A[1][1] = -hp * el.n0n * sC;
  A[2][0] = hp * el.p0V * sC;  A[2][2] = hp * el.p0p * sC;
  B[1][0] = (-hp * el.n1V + hm * er.n0V) * sC;
  B[1][1] = (-hp * el.n1n + hm * er.n0n - fac * dRn_n) * sC;
  B[1][2] = (-fac * dRn_p) * sC;
  B[2][0] = (hp * el.p1V - hm * er.p0V) * sC;
  B[2][1] = (-fac * dRp_n) * sC;
  B[2][2] = (hp * el.p1p - hm * er.p0p - fac * dRp_p) * sC;
  Cm[1][0] = hm * er.n1V * sC; Cm[1][1] = hm * er.n1n * sC;
  Cm[2][0] = -hm * er.p1V * sC; Cm[2][2] = -hm * er.p1p * sC;
  if (ifk_m >= 0 || ifk_i >= 0) {
    const double sc3[3] = {Q * sP, -fac * sC, -fac * sC};
    double Xs[3] = {0.0, 0.0, 0.0};
    Iface t;
    const int lo[3] = {4, 0, 2}, hi[3] = {4, 1, 3};
    if (ifk_m >= 0) {  // the interval behind: its right point is this one
      if (STEADY) iface_edge(L, ifk_m, pm.c.n, pc.c.n, pm.c.p, pc.c.p, t, true);
      else iface_edge_t(L, ifk_m, pm.c.n, pc.c.n, pm.c.p, pc.c.p, fim, dti, t, true, nullptr);
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const int e = hi[q];
        Xs[q] += t.v[e];
        B[q][1] += sc3[q] * t.d[1][e]; B[q][2] += sc3[q] * t.d[3][e];
        A[q][1] += sc3[q] * t.d[0][e]; A[q][2] += sc3[q] * t.d[2][e];
      }
    }
    if (ifk_i >= 0) {  // the interval ahead: its left point is this one
      if (STEADY) iface_edge(L, ifk_i, pc.c.n, pn.c.n, pc.c.p, pn.c.p, t, true);
      else iface_edge_t(L, ifk_i, pc.c.n, pn.c.n, pc.c.p, pn.c.p, fii, dti, t, true, nullptr);
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const int e = lo[q];
        Xs[q] += t.v[e];
        B[q][1] += sc3[q] * t.d[0][e]; B[q][2] += sc3[q] * t.d[2][e];
        Cm[q][1] += sc3[q] * t.d[1][e]; Cm[q][2] += sc3[q] * t.d[3][e];
      }
    }
    pois += Q * Xs[0];
    elec -= fac * Xs[1];
    hole -= fac * Xs[2];
  }
  // implicit Euler in the control volume (ZimT's Cont_Eq_Elec/Holes)
  elec -= fac * dti * (pc.c.n - bn);
  hole -= fac * dti * (pc.c.p - bpd);
  B[1][1] += -fac * dti * pc.c.n * sC;
  B[2][2] += -fac * dti * pc.c.p * sC;
  r[0] = -pois * sP; r[1] = -elec * sC; r[2] = -hole * sC;
  if (mass) {  // each row's time term on its own unknown per unit of dti (`mass=True`)
    mass[0] = 0.0; mass[1] = -fac * pc.c.n * sC; mass[2] = -fac * pc.c.p * sC;
    mass[3] = 0.0; mass[4] = 0.0;
  }
  // the ions' rows (ZimT's Solve_Neg_Ions / Solve_Pos_Ions)
#pragma unroll
  for (int sp = 0; sp < 2; ++sp) {
    const int col = 3 + sp;
    const double sn = sp == 0 ? -1.0 : 1.0;
    const int slot = sp == 0 ? pc.c.sl.a : pc.c.sl.c;
    const double lcv = sp == 0 ? pc.la : pc.lc;
    if (tang) { tang[sp] = 0.0; tang[2 + sp] = 0.0; }
    if (slot < 0) {  // held at its value (0)
      r[col] = -lcv;
      B[col][col] = 1.0;
      continue;
    }
    const int k = sp == 0 ? slot : L.ka + slot;
    const double ls = logs[k];
    if (!(dti > 0.0)) {  // the steady state: Boltzmann's with the slot's normalisation
      r[col] = -(lcv - ls + sn * pc.c.V * iVt);
      B[col][0] = sn * iVt;
      B[col][col] = 1.0;
      U[col][k] = -1.0;
      continue;
    }
    const double before = sp == 0 ? ba : bc;
    const double prev = before > 0.0 ? before : 1.0;
    const int tf = sp == 0 ? T_MUA : T_MUC;
    const double cl = L.Vt * W.x(i - 1, tf), cr = L.Vt * W.x(i, tf);
    // an interval counts inside the species' regions, never a contact's
    const bool inl = (sp == 0 ? pm.c.sl.a : pm.c.sl.c) >= 0 && i > 1;
    const bool inr = (sp == 0 ? pn.c.sl.a : pn.c.sl.c) >= 0 && i < L.NP;
    const double scl = 1.0 / (prev * (fac * dti + hm * cr + hp * cl));
    const double nl = sp == 0 ? pm.a : pm.c2, nc = sp == 0 ? pc.a : pc.c2;
    const double nr = sp == 0 ? pn.a : pn.c2;
    double flux = 0.0, dVl = 0.0, dVc = 0.0, dVr = 0.0, dll = 0.0, dlc = 0.0, dlr = 0.0;
    if (inl) {
      IonIv f;
      if (ivl) f = ivl[sp];  // the interval's fluxes, carried from the row before
      else ion_iv(sn, (pc.c.V - pm.c.V) * iVt, nl, nc, cl, W.simss, f);
      // anions take -hp F_l, cations +hp F_l
      const double w = sp == 0 ? -hp : hp;
      flux += w * f.F;
      dVl -= w * f.gx * iVt; dVc += w * f.gx * iVt;
      dll += w * f.da; dlc += w * f.db;
    }
    if (inr) {
      IonIv f;
      if (ivr) f = ivr[sp];
      else ion_iv(sn, (pn.c.V - pc.c.V) * iVt, nc, nr, cr, W.simss, f);
      // anions take +hm F_r, cations -hm F_r
      const double w = sp == 0 ? hm : -hm;
      flux += w * f.F;
      dVc -= w * f.gx * iVt; dVr += w * f.gx * iVt;
      dlc += w * f.da; dlr += w * f.db;
    }
    const double els = elogs ? elogs[k] : exp(ls);
    const double value = (flux + fac * dti * (els * before - nc)) * scl;
    r[col] = -value;
    A[col][0] = dVl * scl; B[col][0] = dVc * scl; Cm[col][0] = dVr * scl;
    A[col][col] = dll * scl; Cm[col][col] = dlr * scl;
    B[col][col] = (dlc - fac * dti * nc) * scl;
    U[col][k] = fac * dti * els * before * scl;
    if (mass) mass[col] = -fac * nc * scl;
    if (tang) {
      // the row's derivative in the log of the species' mobility (the flux scales with it, and
      // so does the row's scale) and in the log of its density before the step
      const double den = fac * dti + hm * cr + hp * cl;
      tang[sp] = flux * scl - value * (hm * cr + hp * cl) / den;
      tang[2 + sp] = fac * dti * els * before * scl - value;
    }
  }
}

// M^-1 applied in place to v, M = [[P, Q], [R, S]] by its partition (`_inverse5`): Pi the
// carriers' block's inverse, PiQ = Pi Q, R, Si the inverse of S - R Pi Q.
struct Part {
  double Pi[3][3], PiQ[3][2], R[2][3], Si[2][2];
};

__device__ __forceinline__ void partition(const double (&M)[5][5], Part& f) {
  double P[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) P[a][b] = M[a][b];
  inv3(P, f.Pi);
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
      f.PiQ[a][b] = f.Pi[a][0] * M[0][3 + b] + f.Pi[a][1] * M[1][3 + b] + f.Pi[a][2] * M[2][3 + b];
  double S[2][2];
#pragma unroll
  for (int a = 0; a < 2; ++a) {
#pragma unroll
    for (int b = 0; b < 3; ++b) f.R[a][b] = M[3 + a][b];
#pragma unroll
    for (int b = 0; b < 2; ++b)
      S[a][b] = M[3 + a][3 + b] -
                (M[3 + a][0] * f.PiQ[0][b] + M[3 + a][1] * f.PiQ[1][b] + M[3 + a][2] * f.PiQ[2][b]);
  }
  const double idet = 1.0 / (S[0][0] * S[1][1] - S[0][1] * S[1][0]);
  f.Si[0][0] = S[1][1] * idet; f.Si[0][1] = -S[0][1] * idet;
  f.Si[1][0] = -S[1][0] * idet; f.Si[1][1] = S[0][0] * idet;
}

__device__ __forceinline__ void apply(const Part& f, double (&v)[5]) {
  double yt[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) yt[a] = f.Pi[a][0] * v[0] + f.Pi[a][1] * v[1] + f.Pi[a][2] * v[2];
  double w[2];
#pragma unroll
  for (int a = 0; a < 2; ++a)
    w[a] = v[3 + a] - (f.R[a][0] * yt[0] + f.R[a][1] * yt[1] + f.R[a][2] * yt[2]);
  const double z0 = f.Si[0][0] * w[0] + f.Si[0][1] * w[1];
  const double z1 = f.Si[1][0] * w[0] + f.Si[1][1] * w[1];
#pragma unroll
  for (int a = 0; a < 3; ++a) v[a] = yt[a] - (f.PiQ[a][0] * z0 + f.PiQ[a][1] * z1);
  v[3] = z0;
  v[4] = z1;
}

}  // namespace tr
}  // namespace dd
