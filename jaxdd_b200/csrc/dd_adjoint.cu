// The adjoint of the batched J-V solve on sm_100a: the gradient of a function of the curves with
// respect to the packed inputs (the static record, the per-device scalars, the interface table),
// by implicit differentiation at each converged solution.
//
// What it computes is the reverse-mode derivative jaxdd takes through `_converged`'s custom JVP
// (`_converged_jvp` and `_tangent`, src/jaxdd/batch.py:661-737): at a root of the bordered system
// [[T, U], [W^T, D]] (y, z) of the residual F and the ions' constraints g, the derivative of the
// current J(y; theta) is dJ/dtheta = dJ/dtheta|_y - dJ/dy J^-1 d(F, g)/dtheta, and its reverse form
// solves the transposed system once per voltage,
//     [[T^T, W], [U^T, D^T]] (lambda, mu) = (dJ/dy, 0) Jbar,
// giving thetabar = Jbar dJ/dtheta|_y - lambda^T dF/dtheta - mu^T dg/dtheta. A voltage not converged
// (or not finite) contributes nothing, as jaxdd's `valid` mask (batch.py:686-690). jaxdd transposes
// the blocks and runs its sweep again (`_transposed`, batch.py:606-618); here the transposed
// system is solved with the factors of one forward elimination (T = L U, T^T = U^T L^T).
//
// Devices whose ions are frozen after the pre-bias (`_freeze`, batch.py:859-872) get the frozen
// densities' adjoint summed over their voltages, and one more transposed solve at the pre-bias
// solution carries it back to the inputs (jaxdd differentiates through the pre-bias solve and the
// freeze the same way: both are differentiable in its program).
//
// How: one thread takes one device and a share of its voltages (so that a batch of a few thousand
// devices fills the GPU); each voltage is four passes over the grid: the current's reverse sweep
// (right to left) for dJ/dy, the forward elimination with the transposed substitution U^T w = r,
// the back substitution L^T lambda = w with the Schur complement of the ions' border, and a pass
// that accumulates the residual's and the constraints' input derivatives. The results are added
// into the outputs with atomics (threads of one device share them); the outputs are zeroed first.
// The derivatives of the current follow SIMsalabim's integral form (`_current_parts`,
// batch.py:316-403); devices with the differential form (`currDiffInt = 1`) get NaN outputs.
#include <cuda_runtime.h>
#include <stdint.h>

#include "dd_launch.h"
#include "dd_layout.h"
#include "dd_physics.cuh"
#include "../../include/jaxdd_b200.h"

namespace dd {
namespace adj {

// Scratch words per node of one thread. The current's reverse sweep uses the first 13; the
// elimination then reuses them node by node (the right-hand side of a node is read before that
// node's factors are written over it).
enum {
  R_GV = 0, R_GN, R_GP,          // dJ/dy Jbar, the transposed system's right-hand side
  R_EVN, R_EVP, R_IUN, R_IUP,    // exp(+-Vg/V_T), the integrated recombination
  R_UCN, R_UCP, R_RIN, R_RIP,    // the net recombination per carrier, interface recombination
  R_BRN, R_BRP,                  // the interface recombination's adjoint
};
enum { E_MI = 0, E_A = 9, E_COL = 18 };  // then 3 (1 + K) columns, then K ion columns U

template <int K>
constexpr int words() { return E_COL + 3 * (1 + K) + K; }

struct Args {
  int B, Bp, npmax, ka, kc, simss;
  const double* S;
  const double* C;
  const double* IFt;
  const double* V;
  const int* voff;
  const int* vcnt;
  const uint8_t* ok;
  const double* Jbar;
  const double* states;
  const double* state_logs;
  const double* prebias;
  const double* prebias_logs;
  int nv_max;
  double* Sbar;
  double* Cbar;
  double* Ibar;
  double* FX;      // [np+2][2][Bp] frozen densities
  double* FXbar;   // [np+2][2][Bp] their adjoint
  double* scr;     // [np+2][words][T]
  int T, chunks;
};

// A thread's scratch.
struct Scr {
  double* base;
  int T, slot, nw;
  __device__ __forceinline__ double& at(int k, int f) const {
    return base[((size_t)k * nw + f) * T + slot];
  }
};

// The outputs of one device.
struct Out {
  double* S;
  double* C;
  double* I;
  int Bp, l;
  __device__ __forceinline__ void s(int k, int f, double v) const {
    if (v != 0.0) atomicAdd(S + ((size_t)k * DD_NF + f) * Bp + l, v);
  }
  __device__ __forceinline__ void c(int f, double v) const {
    if (v != 0.0) atomicAdd(C + (size_t)f * Bp + l, v);
  }
  __device__ __forceinline__ void i(int row, int f, double v) const {
    if (v != 0.0) atomicAdd(I + ((size_t)row * DD_NIF + f) * Bp + l, v);
  }
};

template <int K>
__device__ void lane_init(Lane& L, const Args& a, int l) {
  L.S = a.S; L.C = a.C; L.IFt = a.IFt; L.Bp = a.Bp; L.l = l;
  L.ka = a.ka; L.K = K;
  L.Vt = L.sc(C_VT); L.iVt = 1.0 / L.Vt; L.L = L.sc(C_L);
      L.gfrac = L.sc(C_GFRAC);
  L.nfloor = L.sc(C_NFLOOR); L.lognf = log(L.nfloor);   L.NP = (int)L.sc(C_NP);
  L.mid = (int)L.sc(C_MID);
  L.currdiff = L.sc(C_CURRDIFF) > 0.0; L.simss = a.simss;
  // the slots' totals: rows past k_anion + k_cation need not exist in scal
#pragma unroll
  for (int k = 0; k < K; ++k) L.tot[k] = k < a.ka + a.kc ? L.sc(C_TOT0 + k) : 0.0;
  L.FX = a.FX; L.CD = nullptr; L.ncd = 0;
  L.ybuf = 0;
  L.frozen = false;
  L.share = 1.0;
  L.half = 0; L.base = 0; L.mask = 0;
}

// The point k of the state (the contacts at 0 and NP + 1).
template <int K>
__device__ __forceinline__ void point(const Lane& L, int k, double Vint, const double* logs, Pt& P) {
  if (k == 0) contact(L, 0, Vint, P);
  else if (k == L.NP + 1) contact(L, 1, Vint, P);
  else { P.V = *L.y(0, k, 0); P.lnn = *L.y(0, k, 1); P.lnp = *L.y(0, k, 2); }
  pt_fill(L, P, k, logs);
}

// The contacts' adjoints gathered while a point is processed.
struct Bar {
  double V0, VR, nL, pL, nR, pR;  // contact potential (left, right), ln n and ln p at both
};

// The record derivatives of recombination at point k, weight w on R.
__device__ void recomb_bar(const Lane& L, const Out& o, int k, double n, double p, double w) {
  if (w == 0.0) return;
  const double kd = L.st(k, S_KD), ni2 = L.st(k, S_NI2), Nt = L.st(k, S_NT);
  o.s(k, S_KD, w * (n * p - ni2));
  o.s(k, S_NI2, -w * kd);
  if (Nt > 0.0) {
    const double Cn = L.st(k, S_CNT), Cp = L.st(k, S_CPT);
    const double nt0 = L.st(k, S_NT0), pt0 = L.st(k, S_PT0);
    const double den = Cn * (n + nt0) + Cp * (p + pt0);
    const double kk = Nt * Cn * Cp;
    const double srh = kk * (n * p - nt0 * pt0) / den;
    o.s(k, S_NT, w * srh / Nt);
    o.s(k, S_CNT, w * (srh / Cn - srh * (n + nt0) / den));
    o.s(k, S_CPT, w * (srh / Cp - srh * (p + pt0) / den));
    o.s(k, S_NT0, w * (-kk * pt0 - srh * Cn) / den);
    o.s(k, S_PT0, w * (-kk * nt0 - srh * Cp) / den);
  }
}

// The current's reverse sweep: dJ/dy Jbar into the scratch's right-hand side, Jbar dJ/dinputs
// into the outputs, the contacts' part into `cb`.
template <int K>
__device__ void current_bar(const Lane& L, const Scr& w, const Out& o, double Vint,
                            const double* logs, double Jbar, Bar& cb) {
  const int NP = L.NP;
  const double Vt = L.Vt, iVt = L.iVt, gf = L.gfrac, LL = L.L;
  const double sign = -L.left();
  // the interface points' recombination (each trapped interval adds to both its ends)
  for (int k = 0; k <= NP + 1; ++k) {
    w.at(k, R_RIN) = 0.0; w.at(k, R_RIP) = 0.0; w.at(k, R_BRN) = 0.0; w.at(k, R_BRP) = 0.0;
    w.at(k, R_GV) = 0.0; w.at(k, R_GN) = 0.0; w.at(k, R_GP) = 0.0;
  }
  for (int e = 0; e <= NP; ++e) {
    const int t = (int)L.st(e, S_IFK);
    if (t < 0) continue;
    Pt a, b;
    point<K>(L, e, Vint, logs, a);
    point<K>(L, e + 1, Vint, logs, b);
    Iface f;
    iface_edge(L, t, a.n, b.n, a.p, b.p, f, false);
    w.at(e, R_RIN) += f.v[0]; w.at(e + 1, R_RIN) += f.v[1];
    w.at(e, R_RIP) += f.v[2]; w.at(e + 1, R_RIP) += f.v[3];
  }
  // forward: exp(+-Vg/V_T), net recombination, its running integral, single and double integrals,
  // the running sums of the recombination currents
  double sgl[2] = {0.0, 0.0}, dbl[2] = {0.0, 0.0}, Ssum[2] = {0.0, 0.0}, iu[2] = {0.0, 0.0};
  double uc_prev[2] = {0.0, 0.0}, dx_prev = 0.0, hsum = 0.0;
  for (int k = 0; k <= NP; ++k) {
    Pt P;
    point<K>(L, k, Vint, logs, P);
    const double ev[2] = {exp(-(P.V + P.offn) * iVt), exp((P.V + P.offp) * iVt)};
    double uc[2] = {0.0, 0.0};
    if (k >= 1) {
      double R, dRn, dRp;
      recomb(L, k, P.n, P.p, R, dRn, dRp);
      const double g = L.st(k, S_G) * gf;
      uc[0] = R + w.at(k, R_RIN) - g;
      uc[1] = R + w.at(k, R_RIP) - g;
    }
    const double dx = k < NP ? L.st(k, S_DX) : 0.0;
    const double hk = L.st(k, S_H);
    hsum += hk;
    const double mu[2] = {L.st(k, S_MUN), L.st(k, S_MUP)};
    const double wk = 0.5 * (dx_prev + dx);
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      if (k >= 1) iu[c] += 0.5 * dx_prev * (uc_prev[c] + uc[c]);
      sgl[c] += wk * ev[c] / mu[c];
      dbl[c] += wk * ev[c] * iu[c] / mu[c];
      if (k >= 1) Ssum[c] += (c == 0 ? -1.0 : 1.0) * Q * LL * hk * uc[c];
      uc_prev[c] = uc[c];
    }
    w.at(k, R_EVN) = ev[0]; w.at(k, R_EVP) = ev[1];
    w.at(k, R_IUN) = iu[0]; w.at(k, R_IUP) = iu[1];
    w.at(k, R_UCN) = uc[0]; w.at(k, R_UCP) = uc[1];
    dx_prev = dx;
  }
  // the contacts' terms of K and K itself
  Pt P0, PR;
  point<K>(L, 0, Vint, logs, P0);
  point<K>(L, NP + 1, Vint, logs, PR);
  const double dens0[2] = {P0.n, P0.p}, densR[2] = {PR.n, PR.p};
  const double ev0[2] = {exp(-(P0.V + P0.offn) * iVt), exp((P0.V + P0.offp) * iVt)};
  const double evR[2] = {exp(-(PR.V + PR.offn) * iVt), exp((PR.V + PR.offp) * iVt)};
  double Kc[2], Bbar[2], sbar[2], dbar[2];
  // The solve's current is sign sum_c [Q K_c + sum_k h_k (J_c,k - Q K_c) / HSUM]: K's term is
  // not weighted by the spacings (they sum to HSUM), so dJ/dK_c = Q sign.
  const double Kbar = Q * Jbar * sign;
  (void)hsum;
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    const double sn = c == 0 ? -1.0 : 1.0;
    const double Bc = Vt * sn * (densR[c] * evR[c] - dens0[c] * ev0[c]);
    Kc[c] = (Bc - sn * dbl[c]) / sgl[c];
    Bbar[c] = Kbar / sgl[c];
    dbar[c] = -sn * Kbar / sgl[c];
    sbar[c] = -Kc[c] * Kbar / sgl[c];
  }
  // contacts: dens0/densR through ln n, ln p; ev0/evR through the potential and the offsets
  cb.nL += Bbar[0] * Vt * (-1.0) * (-dens0[0] * ev0[0]);
  cb.pL += Bbar[1] * Vt * (1.0) * (-dens0[1] * ev0[1]);
  cb.nR += Bbar[0] * Vt * (-1.0) * (densR[0] * evR[0]);
  cb.pR += Bbar[1] * Vt * (1.0) * (densR[1] * evR[1]);
  {
    const double v0 = -Bbar[0] * dens0[0] * ev0[0], p0 = -Bbar[1] * dens0[1] * ev0[1];
    const double vR = Bbar[0] * densR[0] * evR[0], pR = Bbar[1] * densR[1] * evR[1];
    cb.V0 += v0 + p0; cb.VR += vR + pR;
    o.s(0, S_OFFN, v0); o.s(0, S_OFFP, p0);
    o.s(NP + 1, S_OFFN, vR); o.s(NP + 1, S_OFFP, pR);
  }
  // backward, right to left
  double Bsum = 0.0, IS[2] = {0.0, 0.0};
  double Sk[2] = {Ssum[0], Ssum[1]};
  double Lbar = 0.0, Jtot = 0.0, gfbar = 0.0;
  double a_next = 0.0;
  bool iface_next = false;
  for (int k = NP; k >= 0; --k) {
    const double hk = L.st(k, S_H);
    const double a_k = Jbar * sign * hk / L.Hsum();
    const bool iface_k = L.st(k, S_IFK) > -1.5;
    const double b_k = (iface_k ? 0.0 : a_k) + (iface_next ? a_next : 0.0);
    Bsum += b_k;
    Pt P;
    point<K>(L, k, Vint, logs, P);
    const double ev[2] = {w.at(k, R_EVN), w.at(k, R_EVP)};
    const double iuk[2] = {w.at(k, R_IUN), w.at(k, R_IUP)};
    const double uc[2] = {w.at(k, R_UCN), w.at(k, R_UCP)};
    const double mu[2] = {L.st(k, S_MUN), L.st(k, S_MUP)};
    const double dx = k < NP ? L.st(k, S_DX) : 0.0;
    const double dxm = k > 0 ? L.st(k - 1, S_DX) : 0.0;
    const double wk = 0.5 * (dxm + dx);
    double hbar = 0.0, ucbar[2] = {0.0, 0.0}, Vbar = 0.0, offbar[2] = {0.0, 0.0};
    double Jk[2];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const double sn = c == 0 ? -1.0 : 1.0;
      // J_k = Q K + S_k; with an interface at k its averaged value is J_{k-1} + through_k
      Jk[c] = Q * Kc[c] + Sk[c];
      double Jp = Jk[c];
      if (iface_k) {
        const double ri = (c == 0 ? w.at(k, R_RIN) + w.at(k + 1, R_RIN)
                                  : w.at(k, R_RIP) + w.at(k + 1, R_RIP));
        const double thr = sn * 0.5 * Q * LL * hk * ri;
        const double Jprev = k >= 1 ? Jk[c] - sn * Q * LL * hk * uc[c] : Jk[c];
        Jp = Jprev + thr;
        const double rb = a_k * sn * 0.5 * Q * LL * hk;
        w.at(k, c == 0 ? R_BRN : R_BRP) += rb;
        w.at(k + 1, c == 0 ? R_BRN : R_BRP) += rb;
        hbar += a_k * sn * 0.5 * Q * LL * ri;
        Lbar += a_k * sn * 0.5 * Q * hk * ri;
      }
      Jtot += sign * hk * (Jp - Q * Kc[c]) / L.Hsum();
      hbar += Jbar * sign * (Jp - Q * Kc[c]) / L.Hsum();
      // S_k = sum_{m<=k} sn Q L h_m Uc_m, weighted by the suffix sum of b
      if (k >= 1) {
        ucbar[c] += sn * Q * LL * hk * Bsum;
        hbar += sn * Q * LL * uc[c] * Bsum;
        Lbar += sn * Q * hk * uc[c] * Bsum;
        Sk[c] -= sn * Q * LL * hk * uc[c];
      }
      // single and double integrals
      const double evbar = sbar[c] * wk / mu[c] + dbar[c] * wk * iuk[c] / mu[c];
      const double iubar = dbar[c] * wk * ev[c] / mu[c];
      o.s(k, c == 0 ? S_MUN : S_MUP,
          -(sbar[c] * wk * ev[c] + dbar[c] * wk * ev[c] * iuk[c]) / (mu[c] * mu[c]));
      // the running integral: IS_k = sum_{j>=k} iubar_j; Uc_k sits in edges k-1 and k
      const double IS_next = IS[c];
      IS[c] += iubar;
      if (k >= 1) ucbar[c] += 0.5 * dx * IS_next + 0.5 * dxm * IS[c];
      if (k < NP) {
        const double ev1 = c == 0 ? w.at(k + 1, R_EVN) : w.at(k + 1, R_EVP);
        const double iu1 = c == 0 ? w.at(k + 1, R_IUN) : w.at(k + 1, R_IUP);
        const double uc1 = c == 0 ? w.at(k + 1, R_UCN) : w.at(k + 1, R_UCP);
        const double mu1 = c == 0 ? L.st(k + 1, S_MUN) : L.st(k + 1, S_MUP);
        o.s(k, S_DX, 0.5 * (uc[c] + uc1) * IS_next +
                         sbar[c] * 0.5 * (ev[c] / mu[c] + ev1 / mu1) +
                         dbar[c] * 0.5 * (ev[c] * iuk[c] / mu[c] + ev1 * iu1 / mu1));
      }
      const double dv = evbar * ev[c] * sn * iVt;
      Vbar += dv;
      offbar[c] += dv;
    }
    o.s(k, S_H, hbar);
    if (k == 0) { cb.V0 += Vbar; }
    else {
      w.at(k, R_GV) += Vbar;
      const double Rbar = ucbar[0] + ucbar[1];
      double R, dRn, dRp;
      recomb(L, k, P.n, P.p, R, dRn, dRp);
      w.at(k, R_GN) += Rbar * dRn;
      w.at(k, R_GP) += Rbar * dRp;
      recomb_bar(L, o, k, P.n, P.p, Rbar);
      o.s(k, S_G, -Rbar * gf);
      gfbar -= Rbar * L.st(k, S_G);
      w.at(k, R_BRN) += ucbar[0];
      w.at(k, R_BRP) += ucbar[1];
    }
    o.s(k, S_OFFN, offbar[0]);
    o.s(k, S_OFFP, offbar[1]);
    a_next = a_k;
    iface_next = iface_k;
  }
  o.c(C_HSUM, -Jbar * Jtot / L.Hsum());
  o.c(C_L, Lbar);
  o.c(C_GFRAC, gfbar);
  // the interface recombination's adjoint into dJ/dy and the table
  for (int e = 0; e <= NP; ++e) {
    const int t = (int)L.st(e, S_IFK);
    if (t < 0) continue;
    Pt a, b;
    point<K>(L, e, Vint, logs, a);
    point<K>(L, e + 1, Vint, logs, b);
    Iface f;
    iface_edge(L, t, a.n, b.n, a.p, b.p, f, true);
    const double vb[5] = {w.at(e, R_BRN), w.at(e + 1, R_BRN), w.at(e, R_BRP),
                          w.at(e + 1, R_BRP), 0.0};
    double dn0 = 0.0, dn1 = 0.0, dp0 = 0.0, dp1 = 0.0, vv = 0.0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      dn0 += vb[q] * f.d[0][q]; dn1 += vb[q] * f.d[1][q];
      dp0 += vb[q] * f.d[2][q]; dp1 += vb[q] * f.d[3][q];
      vv += vb[q] * f.v[q];
    }
    if (e >= 1) { w.at(e, R_GN) += dn0; w.at(e, R_GP) += dp0; }
    if (e + 1 <= NP) { w.at(e + 1, R_GN) += dn1; w.at(e + 1, R_GP) += dp1; }
    const double Nt = L.itab(t, I_NT), iw = L.itab(t, I_IW);
    if (Nt > 0.0) o.i(t, I_NT, vv / Nt);
    if (iw > 0.0) o.i(t, I_IW, vv / iw);
  }
}

// The transposed bordered solve and the residual's and constraints' input derivatives at one
// solution: right-hand side (V, ln n, ln p) per node in the scratch (R_GV..R_GP), `zbar` for the
// constraints' rows. Adds -lambda^T dF/dinputs - mu^T dg/dinputs into the outputs and, for a frozen
// device, -lambda^T dF/dFX into FXbar; the contacts' part into `cb`.
template <int K>
__device__ void transposed(const Lane& L, const Scr& w, const Out& o, double Vint,
                           const double* logs, const double* zbar, double* FXbar, Bar& cb) {
  const int NP = L.NP;
  constexpr int NC = 1 + K;
  // ---- forward: assemble, factor, U^T w = r
  double cp[3][3], wp[3][NC];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
#pragma unroll
    for (int c = 0; c < 3; ++c) cp[r][c] = 0.0;
#pragma unroll
    for (int c = 0; c < NC; ++c) wp[r][c] = 0.0;
  }
  double num[K];
#pragma unroll
  for (int k = 0; k < K; ++k) num[k] = 0.0;
  Pt pm, pc, pn;
  point<K>(L, 0, Vint, logs, pm);
  point<K>(L, 1, Vint, logs, pc);
  Flux el, er;
  flux(L, pm, pc, L.st(0, S_MUN), L.st(0, S_MUP), el);
  ion_edge<K>(L, pm, pc, L.st(0, S_H) * L.L, num);
  for (int i = 1; i <= NP; ++i) {
    point<K>(L, i + 1, Vint, logs, pn);
    flux(L, pc, pn, L.st(i, S_MUN), L.st(i, S_MUP), er);
    ion_edge<K>(L, pc, pn, L.st(i, S_H) * L.L, num);
    double A[3][3], Bm[3][3], Cm[3][3], rhs[3], U0[K], W[K];
    assemble_row<K>(L, i, pm, pc, pn, el, er, L.st(i - 1, S_H), L.st(i, S_H),
                    (int)L.st(i - 1, S_IFK), (int)L.st(i, S_IFK), false, false, A, Bm, Cm, rhs,
                    U0, W);
    double M[3][3], Mi[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        M[r][c] = Bm[r][c] - (A[r][0] * cp[0][c] + A[r][1] * cp[1][c] + A[r][2] * cp[2][c]);
    inv3(M, Mi);
    // columns: the right-hand side, then W's K columns (the potential's row only)
    double col[3][NC];
    col[0][0] = w.at(i, R_GV); col[1][0] = w.at(i, R_GN); col[2][0] = w.at(i, R_GP);
#pragma unroll
    for (int k = 0; k < K; ++k) { col[0][1 + k] = W[k]; col[1][1 + k] = 0.0; col[2][1 + k] = 0.0; }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      double t[3];
#pragma unroll
      for (int r = 0; r < 3; ++r)
        t[r] = col[r][c] - (cp[0][r] * wp[0][c] + cp[1][r] * wp[1][c] + cp[2][r] * wp[2][c]);
#pragma unroll
      for (int r = 0; r < 3; ++r) { col[r][c] = t[r]; wp[r][c] = t[r]; }
    }
    // c'_i = M^-1 C
    double cn[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        cn[r][c] = Mi[r][0] * Cm[0][c] + Mi[r][1] * Cm[1][c] + Mi[r][2] * Cm[2][c];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cp[r][c] = cn[r][c];
        w.at(i, E_MI + 3 * r + c) = Mi[r][c];
        w.at(i, E_A + 3 * r + c) = A[r][c];
      }
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int r = 0; r < 3; ++r) w.at(i, E_COL + 3 * c + r) = col[r][c];
#pragma unroll
    for (int k = 0; k < K; ++k) w.at(i, E_COL + 3 * NC + k) = U0[k];
    pm = pc; pc = pn; el = er;
  }
  // ---- backward: L^T lambda = w; U^T Lambda for the Schur complement
  double ln[3][NC], An[3][3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
#pragma unroll
    for (int c = 0; c < NC; ++c) ln[r][c] = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) An[r][c] = 0.0;
  }
  double UL[K][NC];
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int c = 0; c < NC; ++c) UL[k][c] = 0.0;
  for (int i = NP; i >= 1; --i) {
    double Mi[3][3], A[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) { Mi[r][c] = w.at(i, E_MI + 3 * r + c); A[r][c] = w.at(i, E_A + 3 * r + c); }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      double t[3];
#pragma unroll
      for (int r = 0; r < 3; ++r)
        t[r] = w.at(i, E_COL + 3 * c + r) - (An[0][r] * ln[0][c] + An[1][r] * ln[1][c] + An[2][r] * ln[2][c]);
#pragma unroll
      for (int r = 0; r < 3; ++r) ln[r][c] = Mi[0][r] * t[0] + Mi[1][r] * t[1] + Mi[2][r] * t[2];
#pragma unroll
      for (int r = 0; r < 3; ++r) w.at(i, E_COL + 3 * c + r) = ln[r][c];
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const double u = w.at(i, E_COL + 3 * NC + k);
#pragma unroll
      for (int c = 0; c < NC; ++c) UL[k][c] += u * ln[0][c];
    }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) An[r][c] = A[r][c];
  }
  // ---- the border: (D^T - U^T Lambda_W) mu = zbar - U^T Lambda_g
  double mu[K];
  {
    double Ms[K][K], rr[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const double tk = L.total(k);
      const double Dk = tk > 0.0 ? num[k] / tk : 1.0;
#pragma unroll
      for (int j = 0; j < K; ++j) Ms[k][j] = (j == k ? Dk : 0.0) - UL[k][1 + j];
      rr[k] = (zbar ? zbar[k] : 0.0) - UL[k][0];
    }
    small_solve<K>(Ms, rr, mu);
  }
  // ---- the inputs' derivatives: lambda = Lambda_g - Lambda_W mu, row by row
  point<K>(L, 0, Vint, logs, pm);
  point<K>(L, 1, Vint, logs, pc);
  flux(L, pm, pc, L.st(0, S_MUN), L.st(0, S_MUP), el);
  for (int i = 1; i <= NP; ++i) {
    point<K>(L, i + 1, Vint, logs, pn);
    flux(L, pc, pn, L.st(i, S_MUN), L.st(i, S_MUP), er);
    double lam[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      double v = w.at(i, E_COL + r);
#pragma unroll
      for (int k = 0; k < K; ++k) v -= w.at(i, E_COL + 3 * (1 + k) + r) * mu[k];
      lam[r] = v;
    }
    const double hm = L.st(i - 1, S_H), hp = L.st(i, S_H);
    const double facl = L.st(i, S_FACL), facm = L.st(i, S_FACM), facu = L.st(i, S_FACU);
    const double fac = L.st(i, S_FAC), sP = L.st(i, S_SP), sC = L.st(i, S_SC);
    double R, dRn, dRp;
    recomb(L, i, pc.n, pc.p, R, dRn, dRp);
    const double G = L.st(i, S_G), gen = G * L.gfrac;
    double X[3] = {0.0, 0.0, 0.0};
    const int ifm = (int)L.st(i - 1, S_IFK), ifi = (int)L.st(i, S_IFK);
    Iface tm, ti;
    if (ifm >= 0) {
      iface_edge(L, ifm, pm.n, pc.n, pm.p, pc.p, tm, false);
      X[0] += tm.v[4]; X[1] += tm.v[1]; X[2] += tm.v[3];
    }
    if (ifi >= 0) {
      iface_edge(L, ifi, pc.n, pn.n, pc.p, pn.p, ti, false);
      X[0] += ti.v[4]; X[1] += ti.v[0]; X[2] += ti.v[2];
    }
    const double afix = L.afix(i), cfix = L.cfix(i);
    const double pois = facl * pm.V + facm * pc.V + facu * pn.V -
                        Q * (pc.n - pc.p + L.st(i, S_DOP) + afix + pc.da - cfix - pc.dc) + Q * X[0];
    const double elec = hm * er.Fn - hp * el.Fn + fac * (gen - R) - fac * X[1];
    const double hole = hp * el.Fp - hm * er.Fp + fac * (gen - R) - fac * X[2];
    // weights on the unscaled rows (every term below is -lambda dF/dinput)
    const double lV = -lam[0] * sP, ln_ = -lam[1] * sC, lp = -lam[2] * sC;
    o.s(i, S_SP, -lam[0] * pois);
    o.s(i, S_SC, -lam[1] * elec - lam[2] * hole);
    o.s(i, S_FACL, lV * pm.V);
    o.s(i, S_FACM, lV * pc.V);
    o.s(i, S_FACU, lV * pn.V);
    o.s(i, S_DOP, -Q * lV);
    if (L.frozen) {
      if (FXbar) {
        atomicAdd(FXbar + ((size_t)i * 2) * L.Bp + L.l, -Q * lV);
        atomicAdd(FXbar + ((size_t)i * 2 + 1) * L.Bp + L.l, Q * lV);
      }
    } else {
      o.s(i, S_AFIX, -Q * lV * L.share);
      o.s(i, S_CFIX, Q * lV * L.share);
    }
    if (i == 1) cb.V0 += lV * facl;
    if (i == NP) cb.VR += lV * facu;
    o.s(i, S_FAC, (ln_ + lp) * (gen - R) - ln_ * X[1] - lp * X[2]);
    o.s(i, S_G, (ln_ + lp) * fac * L.gfrac);
    o.c(C_GFRAC, (ln_ + lp) * fac * G);
    recomb_bar(L, o, i, pc.n, pc.p, -(ln_ + lp) * fac);
    // the fluxes: edge i-1 (el) with weights -hp ln_, hp lp; edge i (er) with hm ln_, -hm lp
    const double wn_el = -hp * ln_, wp_el = hp * lp, wn_er = hm * ln_, wp_er = -hm * lp;
    o.s(i - 1, S_H, ln_ * er.Fn - lp * er.Fp);
    o.s(i, S_H, -ln_ * el.Fn + lp * el.Fp);
    const double mun_m = L.st(i - 1, S_MUN), mup_m = L.st(i - 1, S_MUP);
    const double mun_i = L.st(i, S_MUN), mup_i = L.st(i, S_MUP);
    o.s(i - 1, S_MUN, wn_el * el.Fn / mun_m);
    o.s(i - 1, S_MUP, wp_el * el.Fp / mup_m);
    o.s(i, S_MUN, wn_er * er.Fn / mun_i);
    o.s(i, S_MUP, wp_er * er.Fp / mup_i);
    // offsets enter a flux as its two points' potentials do
    o.s(i - 1, S_OFFN, wn_el * el.n0V);
    o.s(i, S_OFFN, wn_el * el.n1V + wn_er * er.n0V);
    o.s(i + 1, S_OFFN, wn_er * er.n1V);
    o.s(i - 1, S_OFFP, wp_el * el.p0V);
    o.s(i, S_OFFP, wp_el * el.p1V + wp_er * er.p0V);
    o.s(i + 1, S_OFFP, wp_er * er.p1V);
    if (i == 1) {
      cb.V0 += wn_el * el.n0V + wp_el * el.p0V;
      cb.nL += wn_el * el.n0n;
      cb.pL += wp_el * el.p0p;
    }
    if (i == NP) {
      cb.VR += wn_er * er.n1V + wp_er * er.p1V;
      cb.nR += wn_er * er.n1n;
      cb.pR += wp_er * er.p1p;
    }
    // interface traps: every value is proportional to N_t iw
    if (ifm >= 0) {
      const double vv = Q * lV * tm.v[4] - fac * ln_ * tm.v[1] - fac * lp * tm.v[3];
      const double Nt = L.itab(ifm, I_NT), iw = L.itab(ifm, I_IW);
      if (Nt > 0.0) o.i(ifm, I_NT, vv / Nt);
      if (iw > 0.0) o.i(ifm, I_IW, vv / iw);
      if (i == 1) {  // a trapped first interval reaches the left contact's densities
        Iface d;
        iface_edge(L, ifm, pm.n, pc.n, pm.p, pc.p, d, true);
        cb.nL += Q * lV * d.d[0][4] - fac * ln_ * d.d[0][1] - fac * lp * d.d[0][3];
        cb.pL += Q * lV * d.d[2][4] - fac * ln_ * d.d[2][1] - fac * lp * d.d[2][3];
      }
    }
    if (ifi >= 0) {
      const double vv = Q * lV * ti.v[4] - fac * ln_ * ti.v[0] - fac * lp * ti.v[2];
      const double Nt = L.itab(ifi, I_NT), iw = L.itab(ifi, I_IW);
      if (Nt > 0.0) o.i(ifi, I_NT, vv / Nt);
      if (iw > 0.0) o.i(ifi, I_IW, vv / iw);
      if (i == NP) {
        Iface d;
        iface_edge(L, ifi, pc.n, pn.n, pc.p, pn.p, d, true);
        cb.nR += Q * lV * d.d[1][4] - fac * ln_ * d.d[1][0] - fac * lp * d.d[1][2];
        cb.pR += Q * lV * d.d[3][4] - fac * ln_ * d.d[3][0] - fac * lp * d.d[3][2];
      }
    }
    pm = pc; pc = pn; el = er;
  }
  // ---- the constraints: g_k = number_k / total_k - 1 over the intervals of slot k
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const double tk = L.total(k);
    if (!(tk > 0.0) || mu[k] == 0.0) continue;
    o.c(C_TOT0 + k, mu[k] * num[k] / (tk * tk) * L.share);
    o.c(C_L, -mu[k] * num[k] / (L.L * tk));
  }
  {
    Pt a, b;
    point<K>(L, 0, Vint, logs, a);
    for (int e = 0; e <= NP; ++e) {
      point<K>(L, e + 1, Vint, logs, b);
      double hb = 0.0;
      if (a.sl.a >= 0 && a.sl.a == b.sl.a) {
        const int k = a.sl.a;
        const double tk = L.total(k);
        if (tk > 0.0) {
          hb -= mu[k] * 0.5 * (a.da + b.da) * L.L / tk;
          if (e == 0) cb.V0 -= mu[k] * 0.5 * a.da * L.iVt * L.st(0, S_H) * L.L / tk;
          if (e == NP) cb.VR -= mu[k] * 0.5 * b.da * L.iVt * L.st(NP, S_H) * L.L / tk;
        }
      }
      if (a.sl.c >= 0 && a.sl.c == b.sl.c) {
        const int k = L.ka + a.sl.c;
        const double tk = L.total(k);
        if (tk > 0.0) {
          hb -= mu[k] * 0.5 * (a.dc + b.dc) * L.L / tk;
          if (e == 0) cb.V0 += mu[k] * 0.5 * a.dc * L.iVt * L.st(0, S_H) * L.L / tk;
          if (e == NP) cb.VR += mu[k] * 0.5 * b.dc * L.iVt * L.st(NP, S_H) * L.L / tk;
        }
      }
      o.s(e, S_H, hb);
      a = b;
    }
  }
}

// The contacts' adjoint into the scalars; returns the adjoint of the voltage itself.
__device__ double contacts_out(const Lane& L, const Out& o, const Bar& cb) {
  o.c(C_V0, cb.V0);
  o.c(C_VL, cb.VR);
  o.c(C_LNNL, cb.nL);
  o.c(C_LNPL, cb.pL);
  o.c(C_LNNR, cb.nR);
  o.c(C_LNPR, cb.pR);
  return 0.5 * L.left() * (cb.V0 - cb.VR);
}

__device__ __forceinline__ bool finite_state(const Lane& L, const double* logs) {
  bool ok = true;
  for (int k = 1; k <= L.NP && ok; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) ok = ok && isfinite(*L.y(0, k, c));
  for (int k = 0; k < L.K; ++k) ok = ok && isfinite(logs[k]);
  return ok;
}

// The frozen devices' densities (as `freeze` in the solve) from the pre-bias solution.
template <int K>
__global__ void __launch_bounds__(64) frozen_kernel(Args a) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= a.B) return;
  Lane L;
  lane_init<K>(L, a, l);
  if (!(L.sc(C_PRECOND) > 0.0 && L.sc(C_FIXIONS) > 0.0)) return;
  L.Y = const_cast<double*>(a.prebias);
  double logs[K];
#pragma unroll
  for (int k = 0; k < K; ++k) logs[k] = a.prebias_logs[(size_t)k * a.Bp + l];
  for (int i = 1; i <= L.NP; ++i) {
    Pt P;
    point<K>(L, i, 0.0, logs, P);
    a.FX[((size_t)i * 2) * a.Bp + l] = L.st(i, S_AFIX) + P.da;
    a.FX[((size_t)i * 2 + 1) * a.Bp + l] = L.st(i, S_CFIX) + P.dc;
  }
}

// Every converged voltage of every device: thread t takes device t % Bp and its voltages
// t / Bp, t / Bp + chunks, ...
template <int K>
__global__ void __launch_bounds__(64) points_kernel(Args a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.T) return;
  const int l = t % a.Bp, chunk = t / a.Bp;
  if (l >= a.B) return;
  Lane L;
  lane_init<K>(L, a, l);
  const Out o{a.Sbar, a.Cbar, a.Ibar, a.Bp, l};
  if (L.currdiff) {
    if (chunk == 0) o.c(C_VT, NAN);  // the differential current is not differentiated
    return;
  }
  L.frozen = L.sc(C_PRECOND) > 0.0 && L.sc(C_FIXIONS) > 0.0;
  const Scr w{a.scr, a.T, t, words<K>()};
  const int voff = a.voff[l], nv = a.vcnt[l];
  const size_t sstride = (size_t)(a.npmax + 2) * 3 * a.Bp;
  for (int j = chunk; j < nv && j < a.nv_max; j += a.chunks) {
    const int pos = voff + j;
    const double Jb = a.Jbar[pos];
    if (!a.ok[pos] || Jb == 0.0) continue;
    L.Y = const_cast<double*>(a.states) + (size_t)j * sstride;
    double logs[K];
#pragma unroll
    for (int k = 0; k < K; ++k) logs[k] = a.state_logs[((size_t)j * DD_MAXK + k) * a.Bp + l];
    if (!finite_state(L, logs)) continue;
    const double Vint = a.V[pos];
    Bar cb{0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    current_bar<K>(L, w, o, Vint, logs, Jb, cb);
    o.c(C_GSHUNT, Jb * Vint);
    transposed<K>(L, w, o, Vint, logs, nullptr, a.FXbar, cb);
    contacts_out(L, o, cb);
  }
}

// The frozen devices' last transposed solve, at the pre-bias solution: the frozen densities'
// adjoint carried back through the freeze and the pre-bias solve.
template <int K>
__global__ void __launch_bounds__(64) prebias_kernel(Args a) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= a.B) return;
  Lane L;
  lane_init<K>(L, a, l);
  if (L.currdiff || !(L.sc(C_PRECOND) > 0.0 && L.sc(C_FIXIONS) > 0.0)) return;
  const Out o{a.Sbar, a.Cbar, a.Ibar, a.Bp, l};
  const Scr w{a.scr, a.T, l, words<K>()};
  L.Y = const_cast<double*>(a.prebias);
  double logs[K];
#pragma unroll
  for (int k = 0; k < K; ++k) logs[k] = a.prebias_logs[(size_t)k * a.Bp + l];
  if (!finite_state(L, logs)) return;
  const double Vpre = L.sc(C_VPRE);
  double zbar[K];
#pragma unroll
  for (int k = 0; k < K; ++k) zbar[k] = 0.0;
  bool any = false;
  for (int i = 1; i <= L.NP; ++i) {
    const double fa = a.FXbar[((size_t)i * 2) * a.Bp + l];
    const double fc = a.FXbar[((size_t)i * 2 + 1) * a.Bp + l];
    any = any || fa != 0.0 || fc != 0.0;
    Pt P;
    point<K>(L, i, Vpre, logs, P);
    o.s(i, S_AFIX, fa);
    o.s(i, S_CFIX, fc);
    w.at(i, R_GV) = fa * P.da * L.iVt - fc * P.dc * L.iVt;
    w.at(i, R_GN) = 0.0;
    w.at(i, R_GP) = 0.0;
    if (P.sl.a >= 0) zbar[P.sl.a] += fa * P.da;
    if (P.sl.c >= 0) zbar[L.ka + P.sl.c] += fc * P.dc;
  }
  if (!any) return;
  Bar cb{0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  transposed<K>(L, w, o, Vpre, logs, zbar, nullptr, cb);
  o.c(C_VPRE, contacts_out(L, o, cb));
}

}  // namespace adj
}  // namespace dd

// ======================================================================================== C ABI

namespace {

int adj_slots(const dd_batch* b) { return b->k_anion + b->k_cation <= 2 ? 2 : 4; }

int adj_chunks(const dd_batch* b) {
  // about 256 threads (8 warps) per SM of a B200 (148 SMs)
  const long want = 148L * 256;
  int c = (int)((want + b->lane_stride - 1) / b->lane_stride);
  return c < 1 ? 1 : (c > 64 ? 64 : c);
}

size_t adj_bytes(const dd_batch* b, int* T, int* chunks) {
  const int K = adj_slots(b);
  const int nw = K == 2 ? dd::adj::words<2>() : dd::adj::words<4>();
  *chunks = adj_chunks(b);
  *T = b->lane_stride * *chunks;
  const size_t nodes = (size_t)b->np_max + 2;
  return (nodes * 2 * b->lane_stride * 2 + nodes * nw * (size_t)(*T)) * sizeof(double);
}

}  // namespace

extern "C" {

int dd_adjoint_workspace_bytes(const dd_batch* batch, size_t* bytes) {
  if (!batch || !bytes || batch->n_lanes < 1 || batch->lane_stride < batch->n_lanes ||
      batch->lane_stride % 32 != 0 || batch->np_max < 3)
    return DD_ERR_ARGS;
  int T, chunks;
  *bytes = adj_bytes(batch, &T, &chunks);
  return DD_OK;
}

int dd_adjoint(const dd_batch* batch, const dd_voltages* volts, const dd_opts* opts,
               const uint8_t* converged, const double* J_bar, const double* states,
               const double* state_logs, const double* prebias, const double* prebias_logs,
               int nv_max, double* stat_bar, double* scal_bar, double* iface_bar,
               void* workspace, size_t workspace_bytes, void* stream) {
  if (!batch || !batch->stat || !batch->scal || !batch->iface || !volts || !volts->v ||
      !volts->offset || !volts->count || !opts || !converged || !J_bar || !states ||
      !state_logs || !prebias || !prebias_logs || nv_max < 1 || !stat_bar || !scal_bar ||
      !iface_bar || !workspace)
    return DD_ERR_ARGS;
  if (batch->n_lanes < 1 || batch->lane_stride < batch->n_lanes || batch->lane_stride % 32 != 0 ||
      batch->np_max < 3 || batch->k_anion < 1 || batch->k_cation < 1 ||
      batch->k_anion + batch->k_cation > dd::DD_MAXK)
    return DD_ERR_ARGS;
  if (opts->bernoulli != DD_BERNOULLI_EXACT && opts->bernoulli != DD_BERNOULLI_SIMSS)
    return DD_ERR_ARGS;
  int T, chunks;
  if (workspace_bytes < adj_bytes(batch, &T, &chunks)) return DD_ERR_WORKSPACE;
  const size_t nodes = (size_t)batch->np_max + 2;
  const size_t Bp = batch->lane_stride;
  dd::adj::Args a{};
  a.B = batch->n_lanes; a.Bp = batch->lane_stride; a.npmax = batch->np_max;
  a.ka = batch->k_anion; a.kc = batch->k_cation; a.simss = opts->bernoulli == DD_BERNOULLI_SIMSS;
  a.S = batch->stat; a.C = batch->scal; a.IFt = batch->iface;
  a.V = volts->v; a.voff = volts->offset; a.vcnt = volts->count;
  a.ok = converged; a.Jbar = J_bar; a.states = states; a.state_logs = state_logs;
  a.prebias = prebias; a.prebias_logs = prebias_logs; a.nv_max = nv_max;
  a.Sbar = stat_bar; a.Cbar = scal_bar; a.Ibar = iface_bar;
  double* ws = static_cast<double*>(workspace);
  a.FX = ws;
  a.FXbar = ws + nodes * 2 * Bp;
  a.scr = ws + nodes * 2 * Bp * 2;
  a.T = T; a.chunks = chunks;
  int st = dd::device_status();
  if (st != DD_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(stat_bar, 0, nodes * dd::DD_NF * Bp * sizeof(double), s) != cudaSuccess ||
      cudaMemsetAsync(scal_bar, 0, (dd::DD_NS_BASE + dd::DD_MAXK) * Bp * sizeof(double), s) != cudaSuccess ||
      cudaMemsetAsync(iface_bar, 0, (size_t)dd::DD_MAXIF * dd::DD_NIF * Bp * sizeof(double), s) != cudaSuccess ||
      cudaMemsetAsync(a.FX, 0, nodes * 2 * Bp * 2 * sizeof(double), s) != cudaSuccess)
    return DD_ERR_LAUNCH;
  // one warp a block: the threads spread over the 148 SMs more evenly than in pairs of warps
  const dim3 block(32), lanes((a.Bp + 31) / 32), pts((T + 31) / 32);
  if (adj_slots(batch) == 2) {
    st = dd::launch(dd::adj::frozen_kernel<2>, lanes, block, 0, s, a);
    if (st == DD_OK) st = dd::launch(dd::adj::points_kernel<2>, pts, block, 0, s, a);
    if (st == DD_OK) st = dd::launch(dd::adj::prebias_kernel<2>, lanes, block, 0, s, a);
  } else {
    st = dd::launch(dd::adj::frozen_kernel<4>, lanes, block, 0, s, a);
    if (st == DD_OK) st = dd::launch(dd::adj::points_kernel<4>, pts, block, 0, s, a);
    if (st == DD_OK) st = dd::launch(dd::adj::prebias_kernel<4>, lanes, block, 0, s, a);
  }
  return st;
}

}  // extern "C"
