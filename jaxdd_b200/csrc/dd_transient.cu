// Transients with mobile ions on the GPU: jaxdd's `solve_transient` (src/jaxdd/transient.py:
// 270-465, 537-637) for the product's scope, every device through all its time steps in one
// launch.
//
// What: each step is one Newton solve of implicit Euler with the ions as unknowns of their own,
// (V, ln n, ln p, ln a, ln c) per point (`solver._assemble_ions`, solver.py:1364-1475): 5x5
// block-tridiagonal rows bordered by the ion slots, whose rows are each region's number of ions
// over its total (`_ion_constraints_time`, solver.py:1349-1361). The bulk and interface traps'
// occupations are carried from step to step and solved exactly over each step
// (`_trap_step`, solver.py:594-614); each carrier is captured by the occupation's mean over the
// step. The current adds each density's change to the integral form's integrand, the ions'
// currents region by region and the displacement current (batch.py:302-483). ZimT's main loop
// decides which steps are kept (`failureMode`), and each step's dt is from the last kept one.
//
// How: one thread per device (lane), its state in three lane-interleaved buffers
// [node][5][lane] (kept, the one kept before it, the Newton iterate) whose roles rotate when a
// step is kept. A Newton iteration is four passes over the device's points: assembly and forward
// elimination (each 5x5 block solved by its partition as the reference's `_inverse5`: the
// carriers' 3x3 block by its adjugate, then the ions' 2x2 Schur complement), back substitution
// with the slots' K x K Schur complement, the damped update, and the current at the new iterate.
// The static record is the steady solve's (dd_layout.h); the permittivity and the ions'
// mobilities come as a second per-point record.
#include <cuda_runtime.h>
#include <stdint.h>

#include "dd_launch.h"
#include "dd_layout.h"
#include "dd_physics.cuh"
#include "dd_time.cuh"
#include "../../include/jaxdd_b200.h"

namespace dd {
namespace tr {

struct Args {
  const double* S;
  const double* C;
  const double* IFt;
  const double* X;  // [np+2][DD_NT][Bp]
  int n, Bp, npmax, ka, kc;
  // steps
  int steps, tstride;
  const double* t;
  const double* V;
  const double* G;
  const int32_t* track;
  const int32_t* fmode;
  // start: the steady state at the first step
  const double* y0;     // [np+2][3][Bp]
  const double* logs0;  // [DD_MAXK][Bp]
  double tol;
  int max_iter, simss, zimt, ion_last;
  // workspace
  double* Yb;  // [3][np+2][5][Bp]
  double* FB;  // [np+2][Bp]
  double* FI;  // [np+2][Bp]
  double* CD;  // [np+2][ncd][Bp]
  double* BD;  // [np+2][4][Bp]: the state before the step, as densities
  int ncd;
  // outputs
  double* J;
  double* Jext;
  uint8_t* conv;
  int32_t* iters;
  uint8_t* acc;
  int32_t* stop;
  double* state_out;  // [np+2][5][Bp]
  double* logs_out;   // [DD_MAXK][Bp]
  double* fb_out;     // [np+2][Bp] or nullptr
  double* fi_out;     // [np+2][Bp] or nullptr
  // the integrated current and its tangents in ln N_ion and ln mu_ion (nullptr: none)
  double* Qout;       // [Bp]
  double* dQout;      // [2][Bp]
  double* TY;         // [2][2][np+2][5][Bp]: each tangent of the state, two rotating buffers
  double* TFB;        // [2][np+2][Bp]: of the bulk traps' occupations
  double* TFI;        // [2][np+2][Bp]: of the interface traps'
  // each step's state (nullptr: none) and a given state to start from (nullptr: steady)
  double* prof_state;  // [S][np+2][5][Bp]
  double* prof_fb;     // [S][np+2][Bp]
  double* prof_fi;     // [S][np+2][Bp]
  double* prof_dti;    // [S][Bp]
  const double* init_state;  // [np+2][5][Bp]
  const double* init_fb;     // [np+2][Bp]
  const double* init_fi;     // [np+2][Bp]
  const double* init_scal;   // [4][Bp]: t, V_int, J_ext, dti
  // the internal voltage an unknown of every step (vint): each step's open circuit (same layout
  // as t), each lane's series resistance and its external current at the start
  const uint8_t* oc;
  const double* rser;    // [Bp]
  const double* jext0;   // [Bp]
  double* Vout;          // [S][Bp]: each step's internal voltage (nullptr: not written)
  // ZimT's automatic stop: how two states compare (tolPois, tolDens per lane) and the
  // reference state's V, n, p, a, c on every point
  const double* tolp;    // [Bp]
  const double* told;    // [Bp]
  const int32_t* convv;  // [Bp]: ZimT's convVar (nullptr: 1, the densities)
  const double* tolc;    // [Bp]: tolCurr (A/m^2)
  double* REF;           // [np+2][5][Bp]
  // ZimT's tJFile columns of each step (nullptr: none): each lane's layers' first and last
  // points and the columns [S][7 + 8 nlay][Bp]
  const double* LAY;     // [3][nlay][Bp]: i0, i1, the thickness x[i1] - x[i0]
  int nlay;
  double* COL;
};

// ------------------------------------------------------------------------------------ current

// The current over the step at the iterate (buffer `cur`, contacts at Vint) from the state
// before it (buffer `bef`, contacts at Vbef): `_current_parts` with `tr` (batch.py:316-403) and
// `_ion_currents` (421-483), summed over the intervals as `_current` (302-313). One pass left to
// right: each carrier's integral form by prefix sums (sum_e h_e J_e = q K H + sum_e h_e P_e,
// P_e the prefix of q L w_k U_k; an interface's J the one before it plus its traps'), each ion
// region's the same over its own intervals, and the displacement current.
// The state along a tangent: `buf`'s point plus h times the tangent `tan` (point k's field r at
// (k * tn + r * tf) * Bp + l: tn = 5, tf = 1 for a state's layout), the contacts as they are.
__device__ __forceinline__ void load_pert(const View& W, int buf, const double* tan, double h,
                                          int k, double Vint, TP& P, int tn = 5, int tf = 1) {
  load_point(W, buf, k, Vint, P);
  if (!tan || k == 0 || k == W.L.NP + 1) return;
  const size_t o = (size_t)k * tn * W.L.Bp + W.L.l, f = (size_t)tf * W.L.Bp;
  P.c.V += h * tan[o];
  P.c.lnn += h * tan[o + f];
  P.c.lnp += h * tan[o + 2 * f];
  P.la += h * tan[o + 3 * f];
  P.lc += h * tan[o + 4 * f];
  P.c.n = exp(P.c.lnn);
  P.c.p = exp(P.c.lnp);
  P.a = P.c.sl.a >= 0 ? exp(P.la) : 1.0;
  P.c2 = P.c.sl.c >= 0 ? exp(P.lc) : 1.0;
  P.c.da = P.c.sl.a >= 0 ? P.a : 0.0;
  P.c.dc = P.c.sl.c >= 0 ? P.c2 : 0.0;
}

// The state before the step at point k: its potential from buffer `buf`, its densities from the
// step's before-state record (`W.BD`); the contacts as they are.
__device__ __forceinline__ void load_before(const View& W, int buf, int k, double Vint, TP& P) {
  if (!W.BD || k == 0 || k == W.L.NP + 1) { load_point(W, buf, k, Vint, P); return; }
  const size_t o = (size_t)k * 4 * W.L.Bp + W.L.l;
  P.c.V = *W.y(buf, k, 0);
  P.c.n = W.BD[o];
  P.c.p = W.BD[o + W.L.Bp];
  P.a = W.BD[o + 2 * W.L.Bp];
  P.c2 = W.BD[o + 3 * W.L.Bp];
}

// A perturbation of the current's inputs (PERT): the iterate and the state before the step along
// their tangents, the traps' occupations along theirs, the ions' mobilities scaled by `mus`.
struct Pert {
  const double* tcur;
  const double* tbef;
  const double* tfb;
  const double* tfi;
  double h, mus;
  int tn = 5, tf = 1;  // the strides of `tcur` (load_pert)
};

// The constants of the current's integral form that `current_t` finds in its pass: each
// carrier's and each ion region's K (J_e = q K + the prefix of its steps), which regions count.
template <int K>
struct CurK {
  double kc[2], ki[K];
  int first[K];
  bool counted[K];
};

// The other half's value, and a pair's sum in one order on both halves (half 0's first).
__device__ __forceinline__ double pxchg(unsigned mask, double v) {
  return __shfl_xor_sync(mask, v, 1);
}
__device__ __forceinline__ double psum(unsigned mask, bool top, double v) {
  const double o = pxchg(mask, v);
  return top ? v + o : o + v;
}

template <int K, bool PERT = false, bool SPLIT = false>
__device__ double current_t(const View& W, int cur, double Vint, int bef, double Vbef, double dti,
                            double dti_bef, const double* FB, const double* FI,
                            const Pert* pt = nullptr, CurK<K>* ck = nullptr, bool top = true,
                            unsigned mask = 0u) {
  const Lane& L = W.L;
  const double mus = PERT ? pt->mus : 1.0;
  auto fb_at = [&](int k) {
    const size_t o = (size_t)k * L.Bp + L.l;
    return PERT && pt->tfb ? FB[o] + pt->h * pt->tfb[o] : FB[o];
  };
  auto fi_at = [&](int k) {
    const size_t o = (size_t)k * L.Bp + L.l;
    return PERT && pt->tfi ? FI[o] + pt->h * pt->tfi[o] : FI[o];
  };
  auto load_c = [&](int buf, int k, double Vi, TP& P, bool is_cur) {
    if (PERT) {
      load_pert(W, buf, is_cur ? pt->tcur : pt->tbef, pt->h, k, Vi, P, is_cur ? pt->tn : 5,
                is_cur ? pt->tf : 1);
      if (k == 0 || k == L.NP + 1) {  // a contact's ions follow its neighbour along the tangent
        TP nbp;
        load_pert(W, buf, is_cur ? pt->tcur : pt->tbef, pt->h, k == 0 ? 1 : L.NP, Vi, nbp,
                  is_cur ? pt->tn : 5, is_cur ? pt->tf : 1);
        contact_ions(W, buf, k, is_cur ? dti : dti_bef, P, nullptr, &nbp);
        return;
      }
    } else if (is_cur) load_point(W, buf, k, Vi, P);
    else load_before(W, buf, k, Vi, P);
    contact_ions(W, buf, k, is_cur ? dti : dti_bef, P);
  };
  const int NP = L.NP;
  const double QL = Q * L.L;
  double single[2] = {0, 0}, dbl[2] = {0, 0}, iu[2] = {0, 0}, P[2] = {0, 0}, bH[2] = {0, 0};
  double corr[2] = {0, 0}, dtot = 0.0, disp = 0.0;
  double Uprev[2] = {0, 0}, qprev[2] = {0, 0}, Jd_prev[2] = {0, 0};
  double is[K], idb[K], iiu[K], iP[K], iH[K], isum[K], first_v[K], last_v[K], Jion_prev[K];
  int first_k[K];
  bool have[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    is[k] = idb[k] = iiu[k] = iP[k] = iH[k] = isum[k] = first_v[k] = last_v[k] = 0.0;
    Jion_prev[k] = 0.0;
    first_k[k] = -1;
    have[k] = false;
  }
  // SPLIT (the twisted transient's halves): half 0 the iterations 0 .. E - 1, half 1 E .. NP
  // after two that only carry (the capture and U, q at point E - 1, the fluxes of interval
  // E - 1, whether a region is open at E); their sums joined after the loop
  const int E = (NP + 1) / 2;
  const int e0 = SPLIT && !top ? E : 0, ew = SPLIT && !top ? E - 2 : 0;
  const int e1 = SPLIT && top ? E - 1 : NP;
  bool first_here[K], last_here[K];
#pragma unroll
  for (int k = 0; k < K; ++k) { first_here[k] = false; last_here[k] = false; }
  double Hh = 0.0;  // this half's sum of h
  TP pa, pb, qa, qb;  // pa, pb: the iterate at points e, e+1; qa, qb the state before
  load_c(cur, ew, Vint, pa, true);
  load_c(bef, ew, Vbef, qa, false);
  double Ri_next[2] = {0, 0};  // interface capture at point e from the interval before it
  for (int e = ew; e <= e1; ++e) {
    const bool acc = !SPLIT || e >= e0;
    const int kb = e + 1;
    load_c(cur, kb, Vint, pb, true);
    load_c(bef, kb, Vbef, qb, false);
    const double h = L.st(e, S_H), dx = L.st(e, S_DX);
    const int ifk = (int)L.st(e, S_IFK);
    double tRL[2] = {0, 0}, tRR[2] = {0, 0};
    if (ifk >= 0) {
      Iface t;
      iface_edge_t(L, ifk, pa.c.n, pb.c.n, pa.c.p, pb.c.p, fi_at(e), dti, t, false, nullptr);
      tRL[0] = t.v[0]; tRR[0] = t.v[1]; tRL[1] = t.v[2]; tRR[1] = t.v[3];
    }
    // interface capture at points e and e+1 (point e+1's share of interval e+1 is 0: no two
    // trapped interfaces are neighbours)
    const double Ri_a[2] = {Ri_next[0] + tRL[0], Ri_next[1] + tRL[1]};
    const double Ri_b[2] = {tRR[0], tRR[1]};
    double Ue[2] = {0, 0};  // point e's U (0 on the contacts)
    if (e >= 1) {
      double Rn, Rp, d0, d1, d2, d3;
      bulk_rates(L, e, pa.c.n, pa.c.p, fb_at(e), dti, Rn, Rp, d0, d1, d2, d3);
      const double G = L.st(e, S_G) * L.gfrac;
      Ue[0] = Rn + Ri_a[0] - G + dti * (pa.c.n - qa.c.n);
      Ue[1] = Rp + Ri_a[1] - G + dti * (pa.c.p - qa.c.p);
    }
    Ri_next[0] = Ri_b[0]; Ri_next[1] = Ri_b[1];
    const double width = W.zimt ? h : (e == 0 ? h : 0.5 * (L.st(e - 1, S_H) + h));
    double Jd[2] = {0, 0};
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const double sn = s == 0 ? -1.0 : 1.0;
      const double q = exp(sn * (pa.c.V + (s == 0 ? pa.c.offn : pa.c.offp)) * L.iVt) /
                       L.st(e, s == 0 ? S_MUN : S_MUP);
      if (e >= 1 && acc) {
        // interval e-1 (points e-1, e; e-1 <= NP-1): its trapezoid and the two sums
        const double dxm = L.st(e - 1, S_DX);
        const double iu_e = iu[s] + 0.5 * dxm * (Uprev[s] + Ue[s]);
        single[s] += 0.5 * dxm * (qprev[s] + q);
        dbl[s] += 0.5 * dxm * (qprev[s] * iu[s] + q * iu_e);
        iu[s] = iu_e;
        P[s] += sn * QL * width * Ue[s];
      }
      if (acc) bH[s] += h * P[s];
      const double through = sn * 0.5 * QL * h * (Ri_a[s] + Ri_b[s]);
      if (ifk >= -1 && acc)  // a layer interface: the current before it plus through its traps
        corr[s] += h * (through - (e >= 1 ? sn * QL * width * Ue[s] : 0.0));
      if (L.currdiff) {
        const double Vga = pa.c.V + (s == 0 ? pa.c.offn : pa.c.offp);
        const double Vgb = pb.c.V + (s == 0 ? pb.c.offn : pb.c.offp);
        double Bf, Bb, t1, t2;
        bern_pair(sn * (Vgb - Vga) * L.iVt, L.simss, Bf, Bb, t1, t2);
        const double da = s == 0 ? pa.c.n : pa.c.p, db = s == 0 ? pb.c.n : pb.c.p;
        Jd[s] = sn * Q * L.st(e, s == 0 ? S_MUN : S_MUP) * L.Vt * (db * Bb - da * Bf) / (L.L * h);
        if (acc) dtot += h * (ifk >= -1 ? Jd_prev[s] + through : Jd[s]);
      }
      Uprev[s] = Ue[s];
      qprev[s] = q;
    }
    Jd_prev[0] = Jd[0]; Jd_prev[1] = Jd[1];
    // the displacement current of interval e
    if (acc) {
      disp += W.x(e, T_EPS) * ((pb.c.V - pa.c.V) - (qb.c.V - qa.c.V));
      Hh += h;
    }
    // the ions, region by region: exp(+-V/V_T) at the interval's two points, once
    double exa = 1.0, exb = 1.0, iexa = 1.0, iexb = 1.0;
    if (L.tot[0] > 0.0 || L.tot[K - 1] > 0.0 || (K > 2 && (L.tot[1] > 0.0 || L.tot[2] > 0.0))) {
      exa = exp(pa.c.V * L.iVt); exb = exp(pb.c.V * L.iVt);
      iexa = 1.0 / exa; iexb = 1.0 / exb;
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!(L.tot[k] > 0.0)) continue;
      const bool an = k < L.ka;
      const int sk = an ? k : k - L.ka;
      const double sn = an ? -1.0 : 1.0;
      const bool ina = (an ? pa.c.sl.a : pa.c.sl.c) == sk;
      const bool inb = (an ? pb.c.sl.a : pb.c.sl.c) == sk;
      const double da = an ? pa.a : pa.c2, db = an ? pb.a : pb.c2;
      const double qa_ = an ? qa.a : qa.c2, qb_ = an ? qb.a : qb.c2;
      const double eva = an ? iexa : exa, evb = an ? iexb : exb;
      if (ina && !have[k]) {
        have[k] = true;
        first_k[k] = e;
        first_v[k] = da * eva;
        first_here[k] = acc;
      }
      if (inb && acc) {
        last_v[k] = db * evb;
        last_here[k] = true;
      }
      if (L.currdiff) {
        // each interval's flux (an interface takes the interval's before it), counted inside
        double Bf, Bb, t1, t2;
        bern_pair(sn * (pb.c.V - pa.c.V) * L.iVt, L.simss, Bf, Bb, t1, t2);
        const double Jf = sn * Q * mus * W.x(e, an ? T_MUA : T_MUC) * L.Vt * (db * Bb - da * Bf) /
                          (L.L * h);
        if (ina && inb && acc) isum[k] += h * (ifk >= -1 ? Jion_prev[k] : Jf);
        Jion_prev[k] = Jf;
      } else if (ina && inb && acc) {
        const double mua = mus * W.x(e, an ? T_MUA : T_MUC);
        const double mub = mus * W.x(kb, an ? T_MUA : T_MUC);
        const double qa2 = eva / (mua > 0.0 ? mua : 1.0);
        const double qb2 = evb / (mub > 0.0 ? mub : 1.0);
        const double Ua = dti * (da - qa_), Ub = dti * (db - qb_);
        // the ions' trapezoids take every interval, the last one (to the right contact) too
        const double dxi = e < NP ? dx : h * L.L;
        const double iu_b = iiu[k] + 0.5 * dxi * (Ua + Ub);
        is[k] += 0.5 * dxi * (qa2 + qb2);
        idb[k] += 0.5 * dxi * (qa2 * iiu[k] + qb2 * iu_b);
        iiu[k] = iu_b;
        // J_e = qK + the prefix of the steps; at an interface the interval's before it
        const double stp = e > first_k[k] ? sn * QL * width * Ua : 0.0;
        iP[k] += stp;
        iH[k] += h;
        isum[k] += h * (iP[k] - (ifk >= -1 ? stp : 0.0));
      }
    }
    pa = pb;
    qa = qb;
  }
  if constexpr (SPLIT) {
  // half 1's partial sums to half 0, joined as one pass would have summed them: half 1's
  // running integrals and prefixes began at 0, so half 0's last values shift its sums
  const double oHh = pxchg(mask, Hh);
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const double o_single = pxchg(mask, single[s]), o_dbl = pxchg(mask, dbl[s]);
    const double o_bH = pxchg(mask, bH[s]), o_corr = pxchg(mask, corr[s]);
    if (top) {
      dbl[s] = dbl[s] + (o_dbl + iu[s] * o_single);
      bH[s] = bH[s] + (o_bH + P[s] * oHh);
      single[s] += o_single;
      corr[s] += o_corr;
    }
  }
  {
    const double o_dtot = pxchg(mask, dtot), o_disp = pxchg(mask, disp);
    if (top) { dtot += o_dtot; disp += o_disp; }
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const double o_is = pxchg(mask, is[k]), o_idb = pxchg(mask, idb[k]);
    const double o_iH = pxchg(mask, iH[k]), o_isum = pxchg(mask, isum[k]);
    const double o_fv = pxchg(mask, first_v[k]), o_lv = pxchg(mask, last_v[k]);
    const int flags = (have[k] ? 1 : 0) | (first_here[k] ? 2 : 0) | (last_here[k] ? 4 : 0);
    const int o_flags = __shfl_xor_sync(mask, flags, 1);
    if (top) {
      idb[k] = idb[k] + (o_idb + iiu[k] * o_is);
      isum[k] = isum[k] + (o_isum + iP[k] * o_iH);
      is[k] += o_is;
      iH[k] += o_iH;
      if (!have[k] && (o_flags & 2)) first_v[k] = o_fv;
      if (o_flags & 4) last_v[k] = o_lv;
      have[k] = have[k] || (o_flags & 1);
    }
  }
  }
  const double H = L.Hsum();
  double tot = 0.0;
  // ZimT 5.36's ion currents with several regions: each species' last region's alone
  int last_a = -1, last_c = -1;
#pragma unroll
  for (int k = 0; k < K; ++k)
    if (L.tot[k] > 0.0) {
      if (k < L.ka) last_a = k;
      else last_c = k;
    }
  if (!L.currdiff) {
    Pt c0, cN;
    contact(L, 0, Vint, c0);
    contact(L, 1, Vint, cN);
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const double sn = s == 0 ? -1.0 : 1.0;
      const double off0 = L.st(0, s == 0 ? S_OFFN : S_OFFP);
      const double offN = L.st(NP + 1, s == 0 ? S_OFFN : S_OFFP);
      const double d0 = exp(s == 0 ? c0.lnn : c0.lnp), dN = exp(s == 0 ? cN.lnn : cN.lnp);
      const double Kc = (L.Vt * (sn * dN * exp(sn * (cN.V + offN) * L.iVt) -
                                 sn * d0 * exp(sn * (c0.V + off0) * L.iVt)) - sn * dbl[s]) /
                        single[s];
      tot += Q * Kc * H + bH[s] + corr[s];
      if (ck) ck->kc[s] = Kc;
    }
  } else {
    tot = dtot;
  }
  if (ck) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      ck->counted[k] = L.tot[k] > 0.0 && have[k] &&
                       !(W.ion_last && k != (k < L.ka ? last_a : last_c));
      ck->first[k] = first_k[k];
      const double sn = k < L.ka ? -1.0 : 1.0;
      const double sgl = is[k] > 0.0 ? is[k] : 1.0;
      ck->ki[k] = (L.Vt * sn * (last_v[k] - first_v[k]) - sn * idb[k]) / sgl;
    }
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    if (!(L.tot[k] > 0.0) || !have[k]) continue;
    if (W.ion_last && k != (k < L.ka ? last_a : last_c)) continue;
    const double sn = k < L.ka ? -1.0 : 1.0;
    if (!L.currdiff) {
      const double sgl = is[k] > 0.0 ? is[k] : 1.0;
      const double Kc = (L.Vt * sn * (last_v[k] - first_v[k]) - sn * idb[k]) / sgl;
      tot += Q * Kc * iH[k] + isum[k];
    } else {
      tot += isum[k];
    }
  }
  tot += dti * disp / L.L;
  const double J = -L.left() * tot / H;
  if constexpr (SPLIT) return __shfl_sync(mask, J, threadIdx.x & 30u);  // half 0's, to both
  return J;
}

// ------------------------------------------------------------------------------------ columns
//
// ZimT's tJFile columns of a step (`transient._columns`, transient.py:163-222, from
// `_current_parts`, batch.py:316-403): a second pass over the intervals with the constants of
// `current_t`'s pass forms each interval's current as `_current_parts` does (each carrier's
// q K plus the prefix of its steps, an interface's the interval's before it plus its traps';
// each counted ion region's the same inside it; the displacement current), and from them the
// current's rms deviation over the grid, the minority carriers' currents at the contacts and
// the means; per layer (intervals i0 <= e < i1) the QFLS and, as currents, the generation and
// the direct and bulk recombination averaged over the layer, at its last point the interface
// traps' recombination, and its voltage drop. Columns: errJ, JminLeft, JminRight, JShunt,
// Jnion, Jpion, JD, then per layer QFLS, Jphoto, Jdir, JbulkElec, JbulkHoles, JintElec,
// JintHoles, VL (each nlay wide).
constexpr int COL_MAXL = 8;  // the most layers a device's columns take
constexpr int COL_SCALARS = 7;

template <int K>
__device__ __noinline__ void columns_t(const Args& a, const View& W, int cur, double Vint, int bef,
                                       double Vbef, double dti, double dti_bef, double J,
                                       double J_ext, int step, double* err = nullptr) {
  const Lane& L = W.L;
  const int NP = L.NP, Bp = a.Bp, l = L.l, nl = a.nlay;
  const double* FB = a.FB;
  const double* FI = a.FI;
  CurK<K> ck;
  current_t<K>(W, cur, Vint, bef, Vbef, dti, dti_bef, FB, FI, nullptr, &ck);
  int i0[COL_MAXL], i1[COL_MAXL];
  double qf[COL_MAXL], hs[COL_MAXL], gen[COL_MAXL], dir[COL_MAXL], bn[COL_MAXL], bp[COL_MAXL];
  double jin[COL_MAXL], jip[COL_MAXL], vl[COL_MAXL];
  for (int j = 0; j < COL_MAXL; ++j) {
    i0[j] = j < nl ? (int)a.LAY[(size_t)j * Bp + l] : -1;
    i1[j] = j < nl ? (int)a.LAY[(size_t)(nl + j) * Bp + l] : -1;
    qf[j] = hs[j] = gen[j] = dir[j] = bn[j] = bp[j] = jin[j] = jip[j] = vl[j] = 0.0;
  }
  const double QL = Q * L.L, sg = -L.left();
  TP pa, pb, qa, qb;
  load_point(W, cur, 0, Vint, pa);
  contact_ions(W, cur, 0, dti, pa);
  load_before(W, bef, 0, Vbef, qa);
  contact_ions(W, bef, 0, dti_bef, qa);
  double Ri_next[2] = {0, 0}, P[2] = {0, 0}, Jd_prev[2] = {0, 0}, iP[K], Jion_prev[K];
#pragma unroll
  for (int k = 0; k < K; ++k) { iP[k] = 0.0; Jion_prev[k] = 0.0; }
  double dev2 = 0.0, ja = 0.0, jc = 0.0, jdm = 0.0, jmin_l = 0.0, jmin_r = 0.0, last_tot = 0.0;
  for (int e = 0; e <= NP; ++e) {
    const int kb = e + 1;
    load_point(W, cur, kb, Vint, pb);
    contact_ions(W, cur, kb, dti, pb);
    load_before(W, bef, kb, Vbef, qb);
    contact_ions(W, bef, kb, dti_bef, qb);
    const double h = L.st(e, S_H);
    const int ifk = (int)L.st(e, S_IFK);
    double tRL[2] = {0, 0}, tRR[2] = {0, 0};
    if (ifk >= 0) {
      Iface t;
      iface_edge_t(L, ifk, pa.c.n, pb.c.n, pa.c.p, pb.c.p, FI[(size_t)e * Bp + l], dti, t, false,
                   nullptr);
      tRL[0] = t.v[0]; tRR[0] = t.v[1]; tRL[1] = t.v[2]; tRR[1] = t.v[3];
    }
    const double Ri_a[2] = {Ri_next[0] + tRL[0], Ri_next[1] + tRL[1]};
    const double Ri_b[2] = {tRR[0], tRR[1]};
    double Ue[2] = {0, 0}, Rb[2] = {0, 0};
    if (e >= 1) {
      double d0, d1, d2, d3;
      bulk_rates(L, e, pa.c.n, pa.c.p, FB[(size_t)e * Bp + l], dti, Rb[0], Rb[1], d0, d1, d2, d3);
      const double G = L.st(e, S_G) * L.gfrac;
      Ue[0] = Rb[0] + Ri_a[0] - G + dti * (pa.c.n - qa.c.n);
      Ue[1] = Rb[1] + Ri_a[1] - G + dti * (pa.c.p - qa.c.p);
    }
    const double width = W.zimt ? h : (e == 0 ? h : 0.5 * (L.st(e - 1, S_H) + h));
    double Jc2[2];
#pragma unroll
    for (int s2 = 0; s2 < 2; ++s2) {
      const double sn = s2 == 0 ? -1.0 : 1.0;
      const double stp = e >= 1 ? sn * QL * width * Ue[s2] : 0.0;
      P[s2] += stp;
      const double through = sn * 0.5 * QL * h * (Ri_a[s2] + Ri_b[s2]);
      double Jv;
      if (!L.currdiff) {
        const double pre = Q * ck.kc[s2] + P[s2];
        Jv = ifk >= -1 ? pre - stp + through : pre;
      } else {
        const double Vga = pa.c.V + (s2 == 0 ? pa.c.offn : pa.c.offp);
        const double Vgb = pb.c.V + (s2 == 0 ? pb.c.offn : pb.c.offp);
        double Bf, Bb, t1, t2;
        bern_pair(sn * (Vgb - Vga) * L.iVt, L.simss, Bf, Bb, t1, t2);
        const double da = s2 == 0 ? pa.c.n : pa.c.p, db = s2 == 0 ? pb.c.n : pb.c.p;
        const double Jf = sn * Q * L.st(e, s2 == 0 ? S_MUN : S_MUP) * L.Vt * (db * Bb - da * Bf) /
                          (L.L * h);
        Jv = ifk >= -1 ? Jd_prev[s2] + through : Jf;
        Jd_prev[s2] = Jf;
      }
      Jc2[s2] = sg * Jv;
    }
    // the ions, region by region (counted ones), inside each region's intervals
    double Jion[2] = {0, 0};
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!(L.tot[k] > 0.0)) continue;
      const bool an = k < L.ka;
      const int sk = an ? k : k - L.ka;
      const double sn = an ? -1.0 : 1.0;
      const bool ina = (an ? pa.c.sl.a : pa.c.sl.c) == sk;
      const bool inb = (an ? pb.c.sl.a : pb.c.sl.c) == sk;
      const double da = an ? pa.a : pa.c2, db = an ? pb.a : pb.c2;
      const double qa_ = an ? qa.a : qa.c2;
      double Jv = 0.0;
      if (L.currdiff) {
        double Bf, Bb, t1, t2;
        bern_pair(sn * (pb.c.V - pa.c.V) * L.iVt, L.simss, Bf, Bb, t1, t2);
        const double Jf = sn * Q * W.x(e, an ? T_MUA : T_MUC) * L.Vt * (db * Bb - da * Bf) /
                          (L.L * h);
        Jv = ifk >= -1 ? Jion_prev[k] : Jf;
        Jion_prev[k] = Jf;
      } else {
        const double stp =
            (ina && inb && e > ck.first[k]) ? sn * QL * width * dti * (da - qa_) : 0.0;
        iP[k] += stp;
        const double pre = Q * ck.ki[k] + iP[k];
        Jv = ifk >= -1 ? pre - stp : pre;
      }
      if (ck.counted[k] && ina && inb) Jion[an ? 0 : 1] += sg * Jv;
    }
    const double JD = sg * W.x(e, T_EPS) * ((pb.c.V - pa.c.V) - (qb.c.V - qa.c.V)) * dti /
                      (L.L * h);
    const double total = Jc2[0] + Jc2[1] + Jion[0] + Jion[1] + JD;
    dev2 += (total - J) * (total - J);
    last_tot = total;
    ja += h * Jion[0];
    jc += h * Jion[1];
    jdm += h * JD;
    if (e == 0) jmin_l = pa.c.n < pa.c.p ? Jc2[0] : Jc2[1];
    if (e == NP) jmin_r = pb.c.n < pb.c.p ? Jc2[0] : Jc2[1];
    // per layer: the interval's averages, the points' rates, the interface's at its last point
    const double qfls_a = L.Vt * (pa.c.lnn + pa.c.lnp - log(L.st(e, S_NI2)));
    const double qfls_b = L.Vt * (pb.c.lnn + pb.c.lnp - log(L.st(kb, S_NI2)));
    const double direct = e >= 1 ? L.st(e, S_KD) * (pa.c.n * pa.c.p - L.st(e, S_NI2)) : 0.0;
    const double G = e >= 1 ? L.st(e, S_G) * L.gfrac : 0.0;
    for (int j = 0; j < nl && j < COL_MAXL; ++j) {
      if (i0[j] < 0) continue;  // past the lane's own layers
      if (e >= i0[j] && e < i1[j]) {
        qf[j] += h * 0.5 * (qfls_a + qfls_b);
        hs[j] += h;
        gen[j] += h * G;
        dir[j] += h * direct;
        bn[j] += h * (e >= 1 ? Rb[0] - direct : 0.0);
        bp[j] += h * (e >= 1 ? Rb[1] - direct : 0.0);
      }
      if (e == i0[j]) vl[j] -= pa.c.V;
      if (e == i1[j]) {
        vl[j] += pa.c.V;
        jin[j] += QL * h * Ri_a[0];
        jip[j] += QL * h * Ri_a[1];
      }
      if (e == i1[j] + 1) {
        const double hl = L.st(i1[j], S_H);
        jin[j] += QL * hl * Ri_a[0];
        jip[j] += QL * hl * Ri_a[1];
      }
      if (kb == i1[j] && kb == NP + 1) vl[j] += pb.c.V;
    }
    Ri_next[0] = Ri_b[0];
    Ri_next[1] = Ri_b[1];
    pa = pb;
    qa = qb;
  }
  // the point after a layer's last where that is the right contact: its capture Ri_next
  for (int j = 0; j < nl && j < COL_MAXL; ++j)
    if (i0[j] >= 0 && i1[j] + 1 == NP + 1) {
      const double hl = L.st(i1[j], S_H);
      jin[j] += QL * hl * Ri_next[0];
      jip[j] += QL * hl * Ri_next[1];
    }
  dev2 += (last_tot - J) * (last_tot - J);
  if (err) *err = sqrt(dev2 / (NP + 1));
  if (!a.COL) return;
  const double H = L.Hsum();
  const int ncol = COL_SCALARS + 8 * nl;
  double* out = a.COL + (size_t)step * ncol * Bp + l;
  out[0] = sqrt(dev2 / (NP + 1));
  out[(size_t)1 * Bp] = jmin_l;
  out[(size_t)2 * Bp] = jmin_r;
  out[(size_t)3 * Bp] = J_ext - J;
  out[(size_t)4 * Bp] = ja / H;
  out[(size_t)5 * Bp] = jc / H;
  out[(size_t)6 * Bp] = jdm / H;
  for (int j = 0; j < nl && j < COL_MAXL; ++j) {
    const double norm = hs[j] > 0.0 ? hs[j] : 1.0;
    const double thick = a.LAY[(size_t)(2 * nl + j) * Bp + l];
    double v[8] = {qf[j] / norm, Q * gen[j] / norm * thick, Q * dir[j] / norm * thick,
                   Q * bn[j] / norm * thick, Q * bp[j] / norm * thick, jin[j], jip[j], vl[j]};
#pragma unroll
    for (int c = 0; c < 8; ++c) out[(size_t)(COL_SCALARS + c * nl + j) * Bp] = v[c];
  }
}

// ------------------------------------------------------------------------------------ tangents
//
// The integrated current's derivatives in ln N_ion (both species' totals) and ln mu_ion (both
// species' mobilities), forward mode as jaxdd differentiates its transients (`jax.jvp` through
// each step's `_converged_jvp`, batch.py:661-737, carried from step to step by the state): at
// each kept step the tangent of the converged state solves the step's own bordered system at
// that state, its right-hand side the rows' derivatives along the previous state's and the traps'
// previous occupations' tangents and in the parameter itself (the ions' fluxes in ln mu, each
// region's number against its total in ln N); the traps' occupations carry tangents of their
// own; the current's tangent is the central difference of the current along the full tangent
// (the current is an explicit function of its inputs; the step's solve is differentiated
// exactly).

constexpr double TANGENT_H = 1e-6;  // the current's central-difference step along a tangent
constexpr double VINT_H = 1e-6;  // the vint row's central-difference step (V_T, ln units)

// Step k's solution on every point (V, ln n, ln p, and ln a, ln c where the ions are mobile,
// else 0) and the traps' occupations at its end from the ones before it, kept or not
// (`snapshot(after)`, `fb_new`, `fi_new`, transient.py:444): out of line, so that the step
// loop's registers stay its own.
__device__ __noinline__ void write_profile(const Args& a, const View& W, int bn, int k,
                                           double V_k, double dti) {
  const Lane& L = W.L;
  const int NP = L.NP, Bp = a.Bp, l = L.l;
  const size_t nodes = (size_t)a.npmax + 2;
  TP pa, pb;
  load_point(W, bn, 0, V_k, pa);
  for (int i = 0; i <= NP + 1; ++i) {
    TP P;
    load_point(W, bn, i, V_k, P);
    contact_ions(W, bn, i, dti, P);
    const double v5[5] = {P.c.V, P.c.lnn, P.c.lnp, P.c.sl.a >= 0 ? P.la : 0.0,
                          P.c.sl.c >= 0 ? P.lc : 0.0};
#pragma unroll
    for (int c = 0; c < 5; ++c) a.prof_state[(((size_t)k * nodes + i) * 5 + c) * Bp + l] = v5[c];
    a.prof_fb[((size_t)k * nodes + i) * Bp + l] =
        (i >= 1 && i <= NP && L.st(i, S_NT) > 0.0)
            ? bulk_end(L, i, P.c.n, P.c.p, a.FB[(size_t)i * Bp + l], dti)
            : 0.0;
  }
  for (int e = 0; e <= NP; ++e) {
    load_point(W, bn, e + 1, V_k, pb);
    const int ifk = (int)L.st(e, S_IFK);
    double end = 0.0;
    if (ifk >= 0) {
      Iface t;
      iface_edge_t(L, ifk, pa.c.n, pb.c.n, pa.c.p, pb.c.p, a.FI[(size_t)e * Bp + l], dti, t,
                   false, &end);
    }
    a.prof_fi[((size_t)k * nodes + e) * Bp + l] = end;
    pa = pb;
  }
  a.prof_fi[((size_t)k * nodes + NP + 1) * Bp + l] = 0.0;
  a.prof_dti[(size_t)k * Bp + l] = dti;
}

// The tangent's V_int row (`vint` with gradients): the row's coefficients over the border's
// columns (the K slots, then the voltage: `vint_row`'s, over the tangent sweep's columns 2 ..)
// and, per parameter, its right-hand side: less the row's derivative along the tangent sweep's
// own solution (column p), the state before the step and its V_int along theirs, the traps'
// occupations along theirs and, for ln mu, the ions' mobilities.
template <int K, int NC>
__device__ __noinline__ void vint_tangent_row(const Args& a, const View& W, int bn, int bk,
                                              double Vi, double V_now, double tVb[2], double dti,
                                              double dti_now, bool oc, int tb,
                                              double (&row)[K + 1], double (&res)[2]) {
  const Lane& L = W.L;
  const int NP = L.NP, Bp = a.Bp, l = L.l;
  const size_t nodes = (size_t)a.npmax + 2;
  const double* FB = a.FB;
  const double* FI = a.FI;
  const double Rs = a.rser[l];
  const double eV = VINT_H * L.Vt;
  const double dJV = (current_t<K>(W, bn, Vi + eV, bk, V_now, dti, dti_now, FB, FI) -
                      current_t<K>(W, bn, Vi - eV, bk, V_now, dti, dti_now, FB, FI)) /
                         (2.0 * eV) +
                     L.Gshunt();
#pragma unroll
  for (int q = 0; q < K; ++q) row[q] = 0.0;
  row[K] = oc ? dJV / L.Jscale() : (1.0 + Rs * dJV) * L.iVt;
  res[0] = 0.0;
  res[1] = 0.0;
  const double coef = oc ? 1.0 / L.Jscale() : Rs * L.iVt;
  if (coef == 0.0) return;  // V_int = V_ext: a row of the voltage alone
  for (int c = 0; c < NC; ++c) {
    double m = 0.0;
    for (int i = 1; i <= NP; ++i)
#pragma unroll
      for (int rr = 0; rr < 5; ++rr) {
        const double v = fabs(a.CD[((size_t)i * a.ncd + 25 + rr * NC + c) * Bp + l]);
        m = fmax(m, rr == 0 ? v * L.iVt : v);
      }
    Pert pt;
    pt.tcur = a.CD + (size_t)(25 + c) * Bp;
    pt.tn = a.ncd;
    pt.tf = NC;
    pt.tbef = nullptr;
    pt.tfb = nullptr;
    pt.tfi = nullptr;
    pt.mus = 1.0;
    double hb = 0.0;  // the V_int before the step along its tangent
    if (c < 2) {      // a parameter's column: all its inputs along their tangents
      pt.tbef = a.TY + (size_t)(c * 2 + tb) * nodes * 5 * Bp;
      pt.tfb = a.TFB + (size_t)c * nodes * Bp;
      pt.tfi = a.TFI + (size_t)c * nodes * Bp;
      m = fmax(m, 1.0);
      hb = tVb[c];
    } else if (!(m > 0.0) || !isfinite(m)) {
      continue;  // a zero solution: no change
    }
    const double h = VINT_H / m;
    pt.h = h;
    if (c == 1) pt.mus = exp(h);
    const double Jp = current_t<K, true>(W, bn, Vi, bk, V_now + h * hb, dti, dti_now, FB, FI, &pt);
    pt.h = -h;
    if (c == 1) pt.mus = exp(-h);
    const double Jm = current_t<K, true>(W, bn, Vi, bk, V_now - h * hb, dti, dti_now, FB, FI, &pt);
    const double dJ = coef * (Jp - Jm) / (2.0 * h);
    if (c < 2) res[c] -= dJ;
    else row[c - 2] -= dJ;
  }
}

template <int K, bool VINT>
__device__ __noinline__ void tangent_step(const Args& a, View& W, int bn, int bk, double V_k,
                                          double V_now, double dti, double dti_now, double dt,
                                          const double* lg, int tb, double* dQ,
                                          double (&tV)[2][2], bool oc) {
  const Lane& L = W.L;
  const int NP = L.NP, Bp = a.Bp, l = L.l;
  // the two tangents' right-hand sides, then the K slot columns and, with the internal voltage
  // an unknown, its column (the rows' derivative in V_int: `_system_vint`'s)
  constexpr int NC = 2 + K + (VINT ? 1 : 0);
  constexpr int KV = K + (VINT ? 1 : 0);
  const size_t nodes = (size_t)a.npmax + 2;
  auto cd = [&](int k, int f) -> double* { return a.CD + ((size_t)k * a.ncd + f) * Bp + l; };
  auto ty = [&](int p, int b, int k, int c) -> double* {
    return a.TY + ((((size_t)(p * 2 + b) * nodes + k) * 5 + c) * Bp + l);
  };
  auto tfb = [&](int p, int k) { return a.TFB[((size_t)p * nodes + k) * Bp + l]; };
  auto tfi = [&](int p, int k) { return a.TFI[((size_t)p * nodes + k) * Bp + l]; };
  const double* FB = a.FB;
  const double* FI = a.FI;
  double cpv[5][5], dpv[5][NC];
#pragma unroll
  for (int r = 0; r < 5; ++r) {
#pragma unroll
    for (int c = 0; c < 5; ++c) cpv[r][c] = 0.0;
#pragma unroll
    for (int c = 0; c < NC; ++c) dpv[r][c] = 0.0;
  }
  double gnum[K];
#pragma unroll
  for (int q = 0; q < K; ++q) gnum[q] = 0.0;
  TP pm, pc, pn;
  load_point(W, bn, 0, V_k, pm);
  load_point(W, bn, 1, V_k, pc);
  // a region that reaches a contact: the contact's ions from its neighbour's (their share of the
  // region's number; d ln a / d V of the neighbour in dr_c)
  double dr_c[2] = {0.0, 0.0};
  contact_ions(W, bn, 0, dti, pm, &dr_c[0]);
  Flux el, er;
  flux(L, pm.c, pc.c, L.st(0, S_MUN), L.st(0, S_MUP), el);
  double lnc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};  // [side][species]: the contacts' ln density
  lnc[0][0] = pm.la;
  lnc[0][1] = pm.lc;
  for (int i = 1; i <= NP; ++i) {
    load_point(W, bn, i + 1, V_k, pn);
    if (i == NP) {
      contact_ions(W, bn, NP + 1, dti, pn, &dr_c[1]);
      lnc[1][0] = pn.la;
      lnc[1][1] = pn.lc;
    }
    flux(L, pc.c, pn.c, L.st(i, S_MUN), L.st(i, S_MUP), er);
    const double hm = L.st(i - 1, S_H), hp = L.st(i, S_H);
    const int ifm = (int)L.st(i - 1, S_IFK), ifi = (int)L.st(i, S_IFK);
    const double fb = FB[(size_t)i * Bp + l];
    const double fim = ifm >= 0 ? FI[(size_t)(i - 1) * Bp + l] : 0.0;
    const double fii = ifi >= 0 ? FI[(size_t)i * Bp + l] : 0.0;
    const double bnv = exp(*W.y(bk, i, 1)), bpv = exp(*W.y(bk, i, 2));
    const double bav = pc.c.sl.a >= 0 ? exp(*W.y(bk, i, 3)) : 0.0;
    const double bcv = pc.c.sl.c >= 0 ? exp(*W.y(bk, i, 4)) : 0.0;
    double A[5][5], Bm[5][5], Cm[5][5], r[5], U[5][K], tang[4];
    row5<K>(W, i, pm, pc, pn, el, er, hm, hp, ifm, ifi, dti, fb, fim, fii, bnv, bpv, bav, bcv,
            lg, A, Bm, Cm, r, U, nullptr, tang);
    {
      const double hL = hm * L.L;
      if (pc.c.sl.a >= 0 && pc.c.sl.a == pm.c.sl.a) gnum[pc.c.sl.a] += 0.5 * (pm.a + pc.a) * hL;
      if (pc.c.sl.c >= 0 && pc.c.sl.c == pm.c.sl.c)
        gnum[L.ka + pc.c.sl.c] += 0.5 * (pm.c2 + pc.c2) * hL;
      if (i == NP) {  // the last interval, to the right contact
        const double hLr = hp * L.L;
        if (pc.c.sl.a >= 0 && pc.c.sl.a == pn.c.sl.a) gnum[pc.c.sl.a] += 0.5 * (pc.a + pn.a) * hLr;
        if (pc.c.sl.c >= 0 && pc.c.sl.c == pn.c.sl.c)
          gnum[L.ka + pc.c.sl.c] += 0.5 * (pc.c2 + pn.c2) * hLr;
      }
    }
    // the rows' derivatives along each parameter's tangent
    const double fac = L.st(i, S_FAC), sC = L.st(i, S_SC), sP = L.st(i, S_SP);
    double tr_[2][5];
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      double d[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
      if (dti > 0.0) {
        // the time terms in the state before the step
        d[1] += sC * fac * dti * bnv * *ty(p, tb, i, 1);
        d[2] += sC * fac * dti * bpv * *ty(p, tb, i, 2);
        d[3] += tang[2] * *ty(p, tb, i, 3);
        d[4] += tang[3] * *ty(p, tb, i, 4);
        // the bulk traps through their occupation before the step
        const double Nt = L.st(i, S_NT);
        if (Nt > 0.0) {
          const double Cn = L.st(i, S_CNT), Cp = L.st(i, S_CPT);
          const double nt0 = L.st(i, S_NT0), pt0 = L.st(i, S_PT0);
          TrapStep o;
          trap_step(Cn, Cp, nt0, pt0, pc.c.n, pc.c.p, fb, dti, o);
          const double dRn = -Nt * Cn * o.mf * (pc.c.n + nt0), dRp = Nt * Cp * o.mf * (pc.c.p + pt0);
          d[1] += -sC * fac * dRn * tfb(p, i);
          d[2] += -sC * fac * dRp * tfb(p, i);
        }
        // the interface traps of its two intervals through theirs
#pragma unroll
        for (int side = 0; side < 2; ++side) {
          const int e = side == 0 ? i - 1 : i;
          const int t = side == 0 ? ifm : ifi;
          if (t < 0) continue;
          const double Nt_i = L.itab(t, I_NT);
          if (!(Nt_i > 0.0)) continue;
          const TP& qa = side == 0 ? pm : pc;
          const TP& qb = side == 0 ? pc : pn;
          const double Cn = L.itab(t, I_CN), Cp = L.itab(t, I_CP);
          const double nlo = L.itab(t, I_NT0LO), nhi = L.itab(t, I_NT0HI);
          const double plo = L.itab(t, I_PT0LO), phi = L.itab(t, I_PT0HI);
          const double iw = L.itab(t, I_IW);
          const double hq = L.itab(t, I_CHARGE) * 0.5 * Nt_i * iw;
          TrapStep o;
          trap_step(Cn, Cp, nlo + nhi, plo + phi, qa.c.n + qb.c.n, qa.c.p + qb.c.p,
                    side == 0 ? fim : fii, dti, o);
          // this point is the interval's right end (side 0) or its left end (side 1)
          const double nme = side == 0 ? pc.c.n + nhi : pc.c.n + nlo;
          const double pme = side == 0 ? pc.c.p + phi : pc.c.p + plo;
          const double dRn = -iw * Cn * Nt_i * o.mf * nme, dRp = iw * Cp * Nt_i * o.mf * pme;
          const double dQt = -hq * o.Ef;
          const double df = tfi(p, e);
          d[0] += Q * sP * dQt * df;
          d[1] += -fac * sC * dRn * df;
          d[2] += -fac * sC * dRp * df;
        }
      }
      if (p == 1) { d[3] += tang[0]; d[4] += tang[1]; }  // the ions' fluxes in ln mu
#pragma unroll
      for (int c = 0; c < 5; ++c) tr_[p][c] = -d[c];
    }
    double M[5][5];
#pragma unroll
    for (int rr = 0; rr < 5; ++rr)
#pragma unroll
      for (int c = 0; c < 5; ++c) {
        double sm = Bm[rr][c];
#pragma unroll
        for (int q = 0; q < 5; ++q) sm -= A[rr][q] * cpv[q][c];
        M[rr][c] = sm;
      }
    double rhs[5][NC];
#pragma unroll
    for (int rr = 0; rr < 5; ++rr)
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const double uv = (i == 1 ? A[rr][0] * 0.5 * L.left() : 0.0) +
                          (i == NP ? Cm[rr][0] * (-0.5 * L.left()) : 0.0);
        double sm = c < 2 ? tr_[c][rr] : (VINT && c == NC - 1) ? uv : U[rr][c - 2];
#pragma unroll
        for (int q = 0; q < 5; ++q) sm -= A[rr][q] * dpv[q][c];
        rhs[rr][c] = sm;
      }
    Part f;
    partition(M, f);
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      double v[5] = {Cm[0][c], Cm[1][c], Cm[2][c], Cm[3][c], Cm[4][c]};
      apply(f, v);
#pragma unroll
      for (int rr = 0; rr < 5; ++rr) { cpv[rr][c] = v[rr]; *cd(i, rr * 5 + c) = v[rr]; }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      double v[5] = {rhs[0][c], rhs[1][c], rhs[2][c], rhs[3][c], rhs[4][c]};
      apply(f, v);
#pragma unroll
      for (int rr = 0; rr < 5; ++rr) { dpv[rr][c] = v[rr]; *cd(i, 25 + rr * NC + c) = v[rr]; }
    }
    pm = pc;
    pc = pn;
    el = er;
  }
  // back substitution, the slots' Schur complement for both tangents
  double SM[KV][KV], sr[2][KV];
#pragma unroll
  for (int q = 0; q < KV; ++q) {
    const bool has = q < K && L.tot[q] > 0.0;
#pragma unroll
    for (int q2 = 0; q2 < KV; ++q2) SM[q][q2] = (q == q2 && !has) ? 1.0 : 0.0;
    sr[0][q] = has ? gnum[q] / L.tot[q] : 0.0;  // -d g / d ln N: the number over the total
    sr[1][q] = 0.0;
  }
  {
    double xn[5][NC];
#pragma unroll
    for (int rr = 0; rr < 5; ++rr)
#pragma unroll
      for (int c = 0; c < NC; ++c) xn[rr][c] = 0.0;
    Slots s_next = slots_at(L, NP + 1), s_here = slots_at(L, NP);
    for (int i = NP; i >= 1; --i) {
      double xi[5][NC];
#pragma unroll
      for (int rr = 0; rr < 5; ++rr)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          double sm = *cd(i, 25 + rr * NC + c);
#pragma unroll
          for (int q = 0; q < 5; ++q) sm -= *cd(i, rr * 5 + q) * xn[q][c];
          xi[rr][c] = sm;
        }
#pragma unroll
      for (int rr = 0; rr < 5; ++rr)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          *cd(i, 25 + rr * NC + c) = xi[rr][c];
          xn[rr][c] = xi[rr][c];
        }
      const Slots s_prev = slots_at(L, i - 1);
      const double hLm = L.st(i - 1, S_H) * L.L, hLp = L.st(i, S_H) * L.L;
#pragma unroll
      for (int sp = 0; sp < 2; ++sp) {
        const int sl = sp == 0 ? s_here.a : s_here.c;
        if (sl < 0) continue;
        const int q = sp == 0 ? sl : L.ka + sl;
        if (!(L.tot[q] > 0.0)) continue;
        const int slm = sp == 0 ? s_prev.a : s_prev.c, sln = sp == 0 ? s_next.a : s_next.c;
        const double wpt = 0.5 * ((slm == sl ? hLm : 0.0) + (sln == sl ? hLp : 0.0));
        const double w = wpt * exp(*W.y(bn, i, 3 + sp)) / L.tot[q];
        sr[0][q] -= w * xi[3 + sp][0];
        sr[1][q] -= w * xi[3 + sp][1];
#pragma unroll
        for (int q2 = 0; q2 < KV; ++q2) SM[q][q2] -= w * xi[3 + sp][2 + q2];
        // the contact beside this point in the same region: its share of the number follows
        // this point's ln density and potential
        const int side = i == 1 ? 0 : i == NP ? 1 : -1;
        const int slc = side == 0 ? slm : sln;
        if (side >= 0 && slc == sl) {
          const double hLc = side == 0 ? hLm : hLp;
          const double wc = 0.5 * hLc * exp(lnc[side][sp]) / L.tot[q];
          const double wv = wc * (sp == 0 ? dr_c[side] : -dr_c[side]);
          sr[0][q] -= wc * xi[3 + sp][0] + wv * xi[0][0];
          sr[1][q] -= wc * xi[3 + sp][1] + wv * xi[0][1];
#pragma unroll
          for (int q2 = 0; q2 < KV; ++q2) SM[q][q2] -= wc * xi[3 + sp][2 + q2] + wv * xi[0][2 + q2];
        }
      }
      s_next = s_here;
      s_here = s_prev;
    }
  }
  if constexpr (VINT) {  // the voltage's row: its coefficients and, per parameter, its side
    double rowv[K + 1], resv[2];
    double tVb[2] = {tV[0][tb], tV[1][tb]};
    vint_tangent_row<K, NC>(a, W, bn, bk, V_k, V_now, tVb, dti, dti_now, oc, tb, rowv, resv);
#pragma unroll
    for (int q2 = 0; q2 < KV; ++q2) SM[K][q2] = rowv[q2];
    sr[0][K] = resv[0];
    sr[1][K] = resv[1];
  }
  double z[2][KV];
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    double S2[KV][KV];
#pragma unroll
    for (int q = 0; q < KV; ++q)
#pragma unroll
      for (int q2 = 0; q2 < KV; ++q2) S2[q][q2] = SM[q][q2];
    small_solve<KV>(S2, sr[p], z[p]);
    tV[p][1 - tb] = VINT ? z[p][KV - 1] : 0.0;  // the step's V_int along the tangent
  }
  // the state's tangents of this step
  for (int i = 1; i <= NP; ++i)
#pragma unroll
    for (int rr = 0; rr < 5; ++rr) {
#pragma unroll
      for (int p = 0; p < 2; ++p) {
        double v = *cd(i, 25 + rr * NC + p);
#pragma unroll
        for (int q = 0; q < KV; ++q) v -= *cd(i, 25 + rr * NC + 2 + q) * z[p][q];
        *ty(p, 1 - tb, i, rr) = v;
      }
    }
  // the current's tangent: a central difference along the full tangent
  if (dt > 0.0) {
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      Pert pt;
      pt.tcur = a.TY + (size_t)(p * 2 + (1 - tb)) * nodes * 5 * Bp;
      pt.tbef = a.TY + (size_t)(p * 2 + tb) * nodes * 5 * Bp;
      pt.tfb = a.TFB + (size_t)p * nodes * Bp;
      pt.tfi = a.TFI + (size_t)p * nodes * Bp;
      const double hv = TANGENT_H * tV[p][1 - tb], hb = TANGENT_H * tV[p][tb];
      pt.h = TANGENT_H;
      pt.mus = p == 1 ? exp(TANGENT_H) : 1.0;
      const double Jp =
          current_t<K, true>(W, bn, V_k + hv, bk, V_now + hb, dti, dti_now, FB, FI, &pt);
      pt.h = -TANGENT_H;
      pt.mus = p == 1 ? exp(-TANGENT_H) : 1.0;
      const double Jm =
          current_t<K, true>(W, bn, V_k - hv, bk, V_now - hb, dti, dti_now, FB, FI, &pt);
      dQ[p] += (Jp - Jm) / (2.0 * TANGENT_H) * dt;
    }
  }
}

// ------------------------------------------------------------------------------------ kernel

constexpr int MIN_COUNT_STATIC = 5;  // ZimT's equal states in a row that stop a transient
constexpr int STOP_STATIC = 1, STOP_FAILED = 2;

// The state of buffer `buf` (contacts at Vint, their ions at dti) on every point as the
// automatic stop compares states (`summary`, transient.py:361-368): V, n, p and the ions'
// densities where they are mobile, 0 elsewhere.
__device__ __forceinline__ void summary_at(const View& W, int buf, int i, double Vint, double dti,
                                           double (&v)[5]) {
  TP P;
  load_point(W, buf, i, Vint, P);
  contact_ions(W, buf, i, dti, P);
  v[0] = P.c.V; v[1] = P.c.n; v[2] = P.c.p;
  v[3] = P.c.sl.a >= 0 ? P.a : 0.0;
  v[4] = P.c.sl.c >= 0 ? P.c2 : 0.0;
}

// ZimT's `States_Are_Equal` with convVar 1 (transient.py:243-262) of the reference state (REF)
// and the last kept one (buffer `buf`): the potentials within tolPois (the Euclidean norm over
// the grid), each density relatively within tolDens. The generation factors compared apart.
__device__ __noinline__ bool states_equal(const Args& a, const View& W, int buf, double Vint,
                                          double dti, int cv, double dJ, double err) {
  const Lane& L = W.L;
  const int NP = L.NP, Bp = a.Bp, l = L.l;
  double dv = 0.0, d2[4] = {0, 0, 0, 0}, c2[4] = {0, 0, 0, 0}, r2[4] = {0, 0, 0, 0};
  for (int i = 0; i <= NP + 1; ++i) {
    double v[5];
    summary_at(W, buf, i, Vint, dti, v);
    const double* rf = a.REF + (size_t)i * 5 * Bp + l;
    const double e = v[0] - rf[0];
    dv += e * e;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      const double r = rf[(size_t)(f + 1) * Bp], d = v[f + 1] - r;
      d2[f] += d * d;
      c2[f] += v[f + 1] * v[f + 1];
      r2[f] += r * r;
    }
  }
  bool dens = true;
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    const double scale = 0.5 * (sqrt(c2[f]) + sqrt(r2[f]));
    const double rel = scale > 0.0 ? sqrt(d2[f]) / scale : 0.0;
    dens = dens && rel < a.told[l];
  }
  // by convVar: the densities (1), the currents within tolCurr or the smaller errJ (2), either
  // (3), both (4)
  const bool curr = cv != 1 && fabs(dJ) <= fmax(a.tolc[l], err);
  const bool by = cv == 1 ? dens : cv == 2 ? curr : cv == 3 ? (curr || dens) : (curr && dens);
  return sqrt(dv) < a.tolp[l] && by;
}

__device__ __noinline__ void write_ref(const Args& a, const View& W, int buf, double Vint,
                                       double dti) {
  const int NP = W.L.NP, Bp = a.Bp, l = W.L.l;
  for (int i = 0; i <= NP + 1; ++i) {
    double v[5];
    summary_at(W, buf, i, Vint, dti, v);
#pragma unroll
    for (int f = 0; f < 5; ++f) a.REF[((size_t)i * 5 + f) * Bp + l] = v[f];
  }
}

// With the internal voltage an unknown (`vint`), its row of the bordered system (`_vint_row`,
// batch.py:552-563): at the open circuit the external current over the current scale, else
// (V_int + R_series J_ext - V_ext) / V_T, at the iterate. `row` receives its Schur row over the
// border's unknowns (the K slots, then the voltage), `res` its right-hand side less the row's
// product with the sweep's solution of -F. The row's derivatives along the sweep's solutions
// (the columns of CD after the back substitution, dense in the grid) and in V_int are central
// differences of the current, each along a solution scaled to a step of VINT_H (V_T in the
// potential): the reference takes them by reverse-mode autodiff (`jax.value_and_grad`).
template <int K, int NC>
__device__ __noinline__ void vint_row(const Args& a, const View& W, int bn, int bk, double Vi,
                                      double Vext, double V_now, double dti, double dti_now,
                                      bool oc, double (&row)[K + 1], double& res) {
  const Lane& L = W.L;
  const int NP = L.NP, Bp = a.Bp, l = L.l;
  const double* FB = a.FB;
  const double* FI = a.FI;
  const double Rs = a.rser[l];
  const double Je = current_t<K>(W, bn, Vi, bk, V_now, dti, dti_now, FB, FI) + L.Gshunt() * Vi;
  res = -(oc ? Je / L.Jscale() : (Vi + Rs * Je - Vext) * L.iVt);
  const double eV = VINT_H * L.Vt;
  const double dJV = (current_t<K>(W, bn, Vi + eV, bk, V_now, dti, dti_now, FB, FI) -
                      current_t<K>(W, bn, Vi - eV, bk, V_now, dti, dti_now, FB, FI)) /
                         (2.0 * eV) +
                     L.Gshunt();
#pragma unroll
  for (int q = 0; q < K; ++q) row[q] = 0.0;
  row[K] = oc ? dJV / L.Jscale() : (1.0 + Rs * dJV) * L.iVt;
  const double coef = oc ? 1.0 / L.Jscale() : Rs * L.iVt;
  if (coef == 0.0) return;  // V_int = V_ext: a row of the voltage alone
  for (int c = 0; c < NC; ++c) {
    double m = 0.0;
    for (int i = 1; i <= NP; ++i)
#pragma unroll
      for (int rr = 0; rr < 5; ++rr) {
        const double v = fabs(a.CD[((size_t)i * a.ncd + 25 + rr * NC + c) * Bp + l]);
        m = fmax(m, rr == 0 ? v * L.iVt : v);
      }
    if (!(m > 0.0) || !isfinite(m)) continue;  // a zero solution: no change
    Pert pt;
    pt.tcur = a.CD + (size_t)(25 + c) * Bp;
    pt.tbef = nullptr;
    pt.tfb = nullptr;
    pt.tfi = nullptr;
    pt.h = VINT_H / m;
    pt.mus = 1.0;
    pt.tn = a.ncd;
    pt.tf = NC;
    const double Jp = current_t<K, true>(W, bn, Vi, bk, V_now, dti, dti_now, FB, FI, &pt);
    pt.h = -pt.h;
    const double Jm = current_t<K, true>(W, bn, Vi, bk, V_now, dti, dti_now, FB, FI, &pt);
    const double dJ = coef * (Jp - Jm) * m / (2.0 * VINT_H);
    if (c == 0) res -= dJ;
    else row[c - 1] -= dJ;
  }
}

// ------------------------------------------------------------------------------------ twisted
//
// Two threads a device (`transient_kernel<K, false, true>`, neither the internal voltage an
// unknown nor the gradients): the Newton iteration's sweep is twisted as the steady solve's is.
// Half 0 eliminates rows 1 .. m - 1 downwards (c'_i = M_i^-1 C_i, M_i = B_i - A_i c'_{i-1}), half
// 1 rows NP .. m + 1 upwards (a''_i = N_i^-1 A_i, N_i = B_i - C_i a''_{i+1}), each on the same
// code in its own frame (NODE(p) and EDGE(p) walk from its contact inwards); half 0 solves the
// meeting row m, B_m - A_m c'_{m-1} - C_m a''_{m+1}, with half 1's carry, and each half
// substitutes back outwards from x_m. The slots' border and each region's number are summed per
// half and added in one order on both, so both halves solve the same border system. The
// current, the step's start and its end run on half 0 alone.

__device__ __forceinline__ TP tsel(bool t, const TP& x, const TP& y) {
  TP o;
  o.c.V = t ? x.c.V : y.c.V;
  o.c.lnn = t ? x.c.lnn : y.c.lnn;
  o.c.lnp = t ? x.c.lnp : y.c.lnp;
  o.c.n = t ? x.c.n : y.c.n;
  o.c.p = t ? x.c.p : y.c.p;
  o.c.offn = t ? x.c.offn : y.c.offn;
  o.c.offp = t ? x.c.offp : y.c.offp;
  o.c.sl.a = t ? x.c.sl.a : y.c.sl.a;
  o.c.sl.c = t ? x.c.sl.c : y.c.sl.c;
  o.c.da = t ? x.c.da : y.c.da;
  o.c.dc = t ? x.c.dc : y.c.dc;
  o.la = t ? x.la : y.la;
  o.lc = t ? x.lc : y.lc;
  o.a = t ? x.a : y.a;
  o.c2 = t ? x.c2 : y.c2;
  return o;
}

__device__ __forceinline__ Flux fsel(bool t, const Flux& x, const Flux& y) {
  Flux o;
  o.Fn = t ? x.Fn : y.Fn; o.n0V = t ? x.n0V : y.n0V; o.n0n = t ? x.n0n : y.n0n;
  o.n1V = t ? x.n1V : y.n1V; o.n1n = t ? x.n1n : y.n1n; o.Fp = t ? x.Fp : y.Fp;
  o.p0V = t ? x.p0V : y.p0V; o.p0p = t ? x.p0p : y.p0p; o.p1V = t ? x.p1V : y.p1V;
  o.p1p = t ? x.p1p : y.p1p;
  return o;
}

__device__ __forceinline__ IonIv isel(bool t, const IonIv& x, const IonIv& y) {
  return IonIv{t ? x.F : y.F, t ? x.gx : y.gx, t ? x.da : y.da, t ? x.db : y.db};
}

// Each region's number over edge e (points lo = e, hi = e + 1), as the forward pass sums it.
template <int K>
__device__ __forceinline__ void tw_number(const Lane& L, const TP& lo, const TP& hi, int e,
                                          double (&gnum)[K]) {
  const double hL = L.st(e, S_H) * L.L;
  if (hi.c.sl.a >= 0 && hi.c.sl.a == lo.c.sl.a) gnum[hi.c.sl.a] += 0.5 * (lo.a + hi.a) * hL;
  if (hi.c.sl.c >= 0 && hi.c.sl.c == lo.c.sl.c)
    gnum[L.ka + hi.c.sl.c] += 0.5 * (lo.c2 + hi.c2) * hL;
}

// One twisted Newton iteration of a step (no internal voltage): the sweep, the border, the damped
// update of this half's points and the slots' scales `lg`. Returns the step's size and whether the
// new iterate is finite, both of the whole device.
template <int K>
__device__ __forceinline__ void tw_iteration(const Args& a, const View& W, int bn, double Vi,
                                             double dti, double (&lg)[K], bool top,
                                             unsigned mask, double capV, double& size_out,
                                             bool& finite_out) {
  const Lane& L = W.L;
  const int NP = L.NP, Bp = a.Bp, l = L.l;
  constexpr int NC = 1 + K;
  const double* FB = a.FB;
  const double* FI = a.FI;
  auto cd = [&](int k, int f) -> double* { return a.CD + ((size_t)k * a.ncd + f) * Bp + l; };
  const int m = NP / 2;  // the meeting row: half 0 rows 1 .. m, half 1 rows m + 1 .. NP
  const int nown = top ? m : NP - m;
  auto NODE = [&](int p) { return top ? p : NP + 1 - p; };
  auto EDGE = [&](int p) { return top ? p : NP - p; };  // between NODE(p) and NODE(p + 1)
  double cpv[5][5], dpv[5][NC];
#pragma unroll
  for (int r = 0; r < 5; ++r) {
#pragma unroll
    for (int c = 0; c < 5; ++c) cpv[r][c] = 0.0;
#pragma unroll
    for (int c = 0; c < NC; ++c) dpv[r][c] = 0.0;
  }
  double gnum[K], elg[K];
#pragma unroll
  for (int q = 0; q < K; ++q) { gnum[q] = 0.0; elg[q] = exp(lg[q]); }
  // -------- assembly and elimination from this half's contact inwards
  TP po, pc, pi;
  load_point(W, bn, NODE(0), Vi, po);
  contact_ions(W, bn, NODE(0), dti, po);
  load_point(W, bn, NODE(1), Vi, pc);
  Flux fo;
  IonIv ivo[2];
  {
    const TP lo = tsel(top, po, pc), hi = tsel(top, pc, po);
    const int e = EDGE(0);
    flux(L, lo.c, hi.c, L.st(e, S_MUN), L.st(e, S_MUP), fo);
    ion_ivs(W, e, lo, hi, ivo);
    tw_number<K>(L, lo, hi, e, gnum);
  }
  for (int p = 1; p <= nown; ++p) {
    const int i = NODE(p);
    load_point(W, bn, NODE(p + 1), Vi, pi);  // the inner neighbour: inside the device
    const int ei = EDGE(p);
    Flux fi;
    IonIv ivi[2];
    {
      const TP lo = tsel(top, pc, pi), hi = tsel(top, pi, pc);
      flux(L, lo.c, hi.c, L.st(ei, S_MUN), L.st(ei, S_MUP), fi);
      ion_ivs(W, ei, lo, hi, ivi);
      // this half's edges: each point's outer one, and half 0 the meeting row's inner one too
      if (p < nown || top) tw_number<K>(L, lo, hi, ei, gnum);
    }
    // row i in the grid's order: its left and right neighbours and intervals
    const TP pl = tsel(top, po, pi), pr = tsel(top, pi, po);
    const Flux fl = fsel(top, fo, fi), fr = fsel(top, fi, fo);
    IonIv ivl[2], ivr[2];
#pragma unroll
    for (int s = 0; s < 2; ++s) { ivl[s] = isel(top, ivo[s], ivi[s]); ivr[s] = isel(top, ivi[s], ivo[s]); }
    const double hm = L.st(i - 1, S_H), hp = L.st(i, S_H);
    const int ifm = (int)L.st(i - 1, S_IFK), ifi = (int)L.st(i, S_IFK);
    const double fb = FB[(size_t)i * Bp + l];
    const double fim = ifm >= 0 ? FI[(size_t)(i - 1) * Bp + l] : 0.0;
    const double fii = ifi >= 0 ? FI[(size_t)i * Bp + l] : 0.0;
    const size_t ob = (size_t)i * 4 * Bp + l;
    const double bnv = a.BD[ob], bpv = a.BD[ob + Bp];
    const double bav = a.BD[ob + 2 * Bp], bcv = a.BD[ob + 3 * Bp];
    double A[5][5], Bm[5][5], Cm[5][5], r[5], U[5][K];
    row5<K>(W, i, pl, pc, pr, fl, fr, hm, hp, ifm, ifi, dti, fb, fim, fii, bnv, bpv, bav, bcv,
            lg, A, Bm, Cm, r, U, nullptr, nullptr, elg, ivl, ivr);
    if (top && p == nown) {
      // the meeting row waits in memory (the free records of point 0 and of m itself)
#pragma unroll
      for (int rr = 0; rr < 5; ++rr) {
#pragma unroll
        for (int c = 0; c < 5; ++c) {
          *cd(0, rr * 5 + c) = A[rr][c];
          *cd(0, 25 + rr * 5 + c) = Cm[rr][c];
          *cd(m, rr * 5 + c) = Bm[rr][c];
        }
        *cd(m, 25 + rr * NC) = r[rr];
#pragma unroll
        for (int k = 0; k < K; ++k) *cd(m, 25 + rr * NC + 1 + k) = U[rr][k];
      }
    } else {
      // eliminate towards the inside: the outer coupling (A for half 0, C for half 1) against
      // the carry, the inner one into the next carry
      double M[5][5], rhs[5][NC];
#pragma unroll
      for (int rr = 0; rr < 5; ++rr) {
#pragma unroll
        for (int c = 0; c < 5; ++c) {
          double s = Bm[rr][c];
#pragma unroll
          for (int q = 0; q < 5; ++q) s -= (top ? A[rr][q] : Cm[rr][q]) * cpv[q][c];
          M[rr][c] = s;
        }
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          double s = c == 0 ? r[rr] : U[rr][c - 1];
#pragma unroll
          for (int q = 0; q < 5; ++q) s -= (top ? A[rr][q] : Cm[rr][q]) * dpv[q][c];
          rhs[rr][c] = s;
        }
      }
      Part f;
      partition(M, f);
#pragma unroll
      for (int c = 0; c < 5; ++c) {
        double v[5];
#pragma unroll
        for (int rr = 0; rr < 5; ++rr) v[rr] = top ? Cm[rr][c] : A[rr][c];
        apply(f, v);
#pragma unroll
        for (int rr = 0; rr < 5; ++rr) { cpv[rr][c] = v[rr]; *cd(i, rr * 5 + c) = v[rr]; }
      }
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        double v[5] = {rhs[0][c], rhs[1][c], rhs[2][c], rhs[3][c], rhs[4][c]};
        apply(f, v);
#pragma unroll
        for (int rr = 0; rr < 5; ++rr) { dpv[rr][c] = v[rr]; *cd(i, 25 + rr * NC + c) = v[rr]; }
      }
    }
    po = pc;
    pc = pi;
    fo = fi;
    ivo[0] = ivi[0];
    ivo[1] = ivi[1];
  }
  // -------- the meeting row: half 1's carry to half 0, x_m back to half 1
  double oc[5][5], od[5][NC];
#pragma unroll
  for (int r = 0; r < 5; ++r) {
#pragma unroll
    for (int c = 0; c < 5; ++c) oc[r][c] = pxchg(mask, cpv[r][c]);
#pragma unroll
    for (int c = 0; c < NC; ++c) od[r][c] = pxchg(mask, dpv[r][c]);
  }
  double xm[5][NC];
#pragma unroll
  for (int r = 0; r < 5; ++r)
#pragma unroll
    for (int c = 0; c < NC; ++c) xm[r][c] = 0.0;
  if (top) {
    // (B_m - A_m c'_{m-1} - C_m a''_{m+1}) x_m = [r | U]_m - A_m d'_{m-1} - C_m e''_{m+1}
    double G[5][5], R[5][NC];
#pragma unroll
    for (int rr = 0; rr < 5; ++rr) {
#pragma unroll
      for (int c = 0; c < 5; ++c) {
        double s = *cd(m, rr * 5 + c);
#pragma unroll
        for (int q = 0; q < 5; ++q)
          s -= *cd(0, rr * 5 + q) * cpv[q][c] + *cd(0, 25 + rr * 5 + q) * oc[q][c];
        G[rr][c] = s;
      }
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        double s = *cd(m, 25 + rr * NC + c);
#pragma unroll
        for (int q = 0; q < 5; ++q)
          s -= *cd(0, rr * 5 + q) * dpv[q][c] + *cd(0, 25 + rr * 5 + q) * od[q][c];
        R[rr][c] = s;
      }
    }
    Part f;
    partition(G, f);
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      double v[5] = {R[0][c], R[1][c], R[2][c], R[3][c], R[4][c]};
      apply(f, v);
#pragma unroll
      for (int rr = 0; rr < 5; ++rr) { xm[rr][c] = v[rr]; *cd(m, 25 + rr * NC + c) = v[rr]; }
    }
  }
#pragma unroll
  for (int r = 0; r < 5; ++r)
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const double v = pxchg(mask, xm[r][c]);
      if (!top) xm[r][c] = v;
    }
  // -------- back substitution outwards, and this half's part of the border's Schur complement
  // D - W^T X_U and of W^T X_F (each region's number in its points' ion logarithms; where a region
  // reaches a contact, the contact's share in its neighbour's ln density and potential)
  double SMp[K][K], srp[K];
#pragma unroll
  for (int q = 0; q < K; ++q) {
    srp[q] = 0.0;
#pragma unroll
    for (int q2 = 0; q2 < K; ++q2) SMp[q][q2] = 0.0;
  }
  auto border = [&](int i, const double (&xi)[5][NC]) {
    const Slots s_prev = slots_at(L, i - 1), s_here = slots_at(L, i), s_next = slots_at(L, i + 1);
    const double hLm = L.st(i - 1, S_H) * L.L, hLp = L.st(i, S_H) * L.L;
#pragma unroll
    for (int sp = 0; sp < 2; ++sp) {
      const int sl = sp == 0 ? s_here.a : s_here.c;
      if (sl < 0) continue;
      const int q = sp == 0 ? sl : L.ka + sl;
      if (!(L.tot[q] > 0.0)) continue;
      const int slm = sp == 0 ? s_prev.a : s_prev.c, sln = sp == 0 ? s_next.a : s_next.c;
      const double wpt = 0.5 * ((slm == sl ? hLm : 0.0) + (sln == sl ? hLp : 0.0));
      double w = wpt * exp(*W.y(bn, i, 3 + sp)) / L.tot[q], wv = 0.0;
      if ((i == 1 && slm == sl) || (i == NP && sln == sl)) {
        const int kc = i == 1 ? 0 : NP + 1;
        TP P;
        load_point(W, bn, kc, Vi, P);
        double dr;
        contact_ions(W, bn, kc, dti, P, &dr);
        const double wc = 0.5 * (i == 1 ? hLm : hLp) * (sp == 0 ? P.a : P.c2) / L.tot[q];
        w += wc;
        wv = wc * (sp == 0 ? dr : -dr);
      }
      srp[q] += w * xi[3 + sp][0] + wv * xi[0][0];
#pragma unroll
      for (int q2 = 0; q2 < K; ++q2) SMp[q][q2] += w * xi[3 + sp][1 + q2] + wv * xi[0][1 + q2];
    }
  };
  if (top) border(m, xm);
  {
    double xn[5][NC];
#pragma unroll
    for (int rr = 0; rr < 5; ++rr)
#pragma unroll
      for (int c = 0; c < NC; ++c) xn[rr][c] = xm[rr][c];
    for (int p = top ? nown - 1 : nown; p >= 1; --p) {
      const int i = NODE(p);
      double xi[5][NC];
#pragma unroll
      for (int rr = 0; rr < 5; ++rr)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          double s = *cd(i, 25 + rr * NC + c);
#pragma unroll
          for (int q = 0; q < 5; ++q) s -= *cd(i, rr * 5 + q) * xn[q][c];
          xi[rr][c] = s;
        }
#pragma unroll
      for (int rr = 0; rr < 5; ++rr)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          *cd(i, 25 + rr * NC + c) = xi[rr][c];
          xn[rr][c] = xi[rr][c];
        }
      border(i, xi);
    }
  }
  // both halves' parts, and the numbers, added in one order: the same border system on both
  double SM[K][K], sr[K], z[K];
#pragma unroll
  for (int q = 0; q < K; ++q) gnum[q] = psum(mask, top, gnum[q]);
#pragma unroll
  for (int q = 0; q < K; ++q) {
    const bool has = L.tot[q] > 0.0;
    sr[q] = -(has ? gnum[q] / L.tot[q] - 1.0 : lg[q]) - psum(mask, top, srp[q]);
#pragma unroll
    for (int q2 = 0; q2 < K; ++q2)
      SM[q][q2] = ((q == q2 && !has) ? 1.0 : 0.0) - psum(mask, top, SMp[q][q2]);
  }
  small_solve<K>(SM, sr, z);
  // -------- the damped update (batch.py:759-785) of this half's points
  double size = 0.0, dl_max = 0.0;
  bool finite = true;
#pragma unroll
  for (int q = 0; q < K; ++q) {
    const double dlq = clipd(z[q], -ION_LOG_CAP, ION_LOG_CAP);
    dl_max = nanmax(dl_max, fabs(dlq));
    lg[q] += dlq;
  }
  for (int p = 1; p <= nown; ++p) {
    const int i = NODE(p);
    double d5[5];
#pragma unroll
    for (int rr = 0; rr < 5; ++rr) {
      double s = *cd(i, 25 + rr * NC);
#pragma unroll
      for (int q = 0; q < K; ++q) s -= *cd(i, 25 + rr * NC + 1 + q) * z[q];
      d5[rr] = s;
    }
    double y5[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) y5[c] = *W.y(bn, i, c);
    double st5[5];
    st5[0] = clipd(d5[0], -capV, capV);
#pragma unroll
    for (int c = 1; c < 5; ++c) st5[c] = clipd(d5[c], -CAP_LN, CAP_LN);
#pragma unroll
    for (int c = 1; c < 3; ++c) {  // a density below the floor steps in the density
      if (y5[c] < L.lognf) {
        const double dd = d5[c];
        const double in_n = dd > -1.0 ? log1p(dd) : -CAP_LN;
        st5[c] = clipd(in_n, -FLOOR_DROP_CAP, CAP_LN);
      }
    }
    size = nanmax(size, fabs(st5[0]) * L.iVt);
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      const double nw = y5[c] + st5[c];
      *W.y(bn, i, c) = nw;
      finite = finite && isfinite(nw);
      if (c >= 1) {
        const double dens = exp(nw);
        size = nanmax(size, fabs(st5[c]) * (dens / (dens + L.nfloor)));
      }
    }
  }
  size = nanmax(size, pxchg(mask, size));
  size = nanmax(size, dl_max);
  finite = __shfl_xor_sync(mask, finite ? 1 : 0, 1) != 0 && finite;
#pragma unroll
  for (int q = 0; q < K; ++q) finite = finite && isfinite(lg[q]);
  size_out = size;
  finite_out = finite;
  __syncwarp(mask);  // both halves' points written before either reads the other's
}

template <int K, bool VINT, bool TW = false>
__global__ void __launch_bounds__(32) transient_kernel(Args a) {
  // one thread a device, or with TW two (the twisted sweep), half 0 the device's serial parts
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int l = TW ? t >> 1 : t;
  const bool top = !TW || (t & 1) == 0;
  const unsigned mask = TW ? (0x3u << (threadIdx.x & 30u)) : 0xffffffffu;
  if (l >= a.n) return;
  View W;
  Lane& L = W.L;
  L.S = a.S; L.C = a.C; L.IFt = a.IFt; L.Bp = a.Bp; L.l = l;
  L.NP = (int)L.sc(C_NP);
  L.ka = a.ka; L.K = K;
  L.Vt = L.sc(C_VT); L.iVt = 1.0 / L.Vt; L.L = L.sc(C_L);       L.nfloor = L.sc(C_NFLOOR); L.lognf = log(L.nfloor);   L.currdiff = L.sc(C_CURRDIFF) > 0.0; L.simss = a.simss;
  L.frozen = false; L.share = 1.0;
  // the slots' totals: rows past k_anion + k_cation need not exist in scal
#pragma unroll
  for (int k = 0; k < K; ++k) L.tot[k] = k < a.ka + a.kc ? L.sc(C_TOT0 + k) : 0.0;
  W.X = a.X; W.Yb = a.Yb; W.ybuf = (size_t)(a.npmax + 2) * 5 * a.Bp; W.simss = a.simss;
  W.zimt = a.zimt; W.BD = a.BD; W.ion_last = a.ion_last;
  const int NP = L.NP, Bp = a.Bp;
  const int ts = a.tstride;
  double* FB = a.FB;
  double* FI = a.FI;
  auto cd = [&](int k, int f) -> double* { return a.CD + ((size_t)k * a.ncd + f) * Bp + l; };
  // right-hand sides: -F, the K slot columns and with VINT the internal voltage's
  constexpr int NC = VINT ? 2 + K : 1 + K;
  constexpr int KV = VINT ? K + 1 : K;  // the border's unknowns

  // ---- the start: the steady state at the first step, with the ions' densities as unknowns,
  // or a given state (its slots' scales 1)
  int bk = 0, bp = 1, bn = 2;  // kept, kept before it, iterate
  const bool given = a.init_state != nullptr;
  double logs[K], logs_p[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    logs[k] = given ? 0.0 : a.logs0[(size_t)k * Bp + l];
    logs_p[k] = logs[k];
  }
  for (int i = 1; i <= NP && top; ++i) {
    const Slots sl = slots_at(L, i);
    double v5[5];
    if (given) {
#pragma unroll
      for (int c = 0; c < 5; ++c) v5[c] = a.init_state[((size_t)i * 5 + c) * Bp + l];
      if (sl.a < 0) v5[3] = 0.0;
      if (sl.c < 0) v5[4] = 0.0;
    } else {
      const double V = a.y0[((size_t)i * 3 + 0) * Bp + l];
      v5[0] = V;
      v5[1] = a.y0[((size_t)i * 3 + 1) * Bp + l];
      v5[2] = a.y0[((size_t)i * 3 + 2) * Bp + l];
      v5[3] = sl.a >= 0 ? logs[sl.a] + V * L.iVt : 0.0;
      v5[4] = sl.c >= 0 ? logs[L.ka + sl.c] - V * L.iVt : 0.0;
    }
#pragma unroll
    for (int c = 0; c < 5; ++c) { *W.y(bk, i, c) = v5[c]; *W.y(bp, i, c) = v5[c]; }
    FB[(size_t)i * Bp + l] = given ? a.init_fb[(size_t)i * Bp + l] : 0.0;
  }
  for (int e = 0; e <= NP && top; ++e)
    FI[(size_t)e * Bp + l] = given ? a.init_fi[(size_t)e * Bp + l] : 0.0;
  const int fm = a.fmode[l];
  // the integrated current and its tangents (zero tangents before the first step)
  const bool grad = a.TY != nullptr;
  const size_t tnodes = (size_t)a.npmax + 2;
  double Qint = 0.0, dQ[2] = {0.0, 0.0};
  double tVv[2][2] = {{0.0, 0.0}, {0.0, 0.0}};  // V_int along each tangent: [parameter][buffer]
  int tb = 0;
  if (grad) {
    for (int p = 0; p < 4; ++p)
      for (int i = 0; i <= NP + 1; ++i)
#pragma unroll
        for (int c = 0; c < 5; ++c) a.TY[(((size_t)p * tnodes + i) * 5 + c) * Bp + l] = 0.0;
    for (int p = 0; p < 2; ++p)
      for (int i = 0; i <= NP + 1; ++i) {
        a.TFB[((size_t)p * tnodes + i) * Bp + l] = 0.0;
        a.TFI[((size_t)p * tnodes + i) * Bp + l] = 0.0;
      }
  }
  double V_now = given ? a.init_scal[(size_t)Bp + l] : a.V[ts ? l : 0];
  double dti_now = given ? a.init_scal[(size_t)3 * Bp + l] : 0.0;
  double t_last = given ? a.init_scal[l] : 0.0;
  // the internal voltage kept before the last one, and the external current of the last
  double V_before = V_now;
  double J_ext_now = given ? a.init_scal[(size_t)2 * Bp + l] : (VINT ? a.jext0[l] : 0.0);
  int track_curr = 0, stop = 0, count = 0;
  double G_cur = -1.0, G_ref = -1.0;  // the generation factors of the kept and reference states
  // and their currents and errJ, for convVar 2-4
  double J_cur = 0.0, J_ref = 0.0, err_cur = 0.0, err_ref = 0.0;
  const int cv = a.convv && a.tolc ? a.convv[l] : 1;
  bool first = true;
  const double capV = CAP_V * L.Vt;

  for (int k = 0; k < a.steps; ++k) {
    // step k of this lane: one list for all lanes (ts 0) or [step][lane]
    const size_t so = ts ? (size_t)k * ts + l : (size_t)k;
    const double t_k = a.t[so], V_k = a.V[so];
    L.gfrac = a.G[so];
    const double dti = t_k == 0.0 ? 0.0 : 1.0 / (t_k > t_last ? t_k - t_last : 1.0);
    const bool moving = dti > 0.0 && dti_now > 0.0 && !first;
    const double rt = moving ? dti_now / dti : 0.0;
    // the internal voltage of the iterate: given, or with VINT an unknown from the last one at
    // the open circuit (extrapolated as the state), else the external voltage less the last
    // current's drop (transient.py:398-401)
    const bool oc_k = VINT && a.oc[so] != 0;
    double Vi = V_k;
    if (VINT)
      Vi = oc_k ? V_now + clipd(rt * (V_now - V_before), -capV, capV)
                : V_k - a.rser[l] * J_ext_now;
    // ---- the step's start: the last two kept states extrapolated, held to one step's caps;
    // into a steady state the slots' Boltzmann normalisations of it
    double num[K];
#pragma unroll
    for (int q = 0; q < K; ++q) num[q] = 0.0;
    {
      // with TW half 0 points 1 .. m, half 1 m + 1 .. NP + 1 (the point before its first
      // extrapolated again for the numbers' trapezoid)
      const int mh = NP / 2;
      const int lo = TW && !top ? mh + 1 : 1, hi = TW && top ? mh : NP + 1;
      double Vprev = L.V0() + 0.5 * L.left() * Vi;
      if (lo > 1) {
        const double y = *W.y(bk, lo - 1, 0), yp = *W.y(bp, lo - 1, 0);
        Vprev = y + clipd(rt * (y - yp), -capV, capV);
      }
      Slots slp = slots_at(L, lo - 1);
      for (int i = lo; i <= hi; ++i) {
        double V;
        if (i <= NP) {
#pragma unroll
          for (int c = 0; c < 5; ++c) {
            const double y = *W.y(bk, i, c), yp = *W.y(bp, i, c);
            const double cap = c == 0 ? capV : CAP_LN;
            *W.y(bn, i, c) = y + clipd(rt * (y - yp), -cap, cap);
          }
          // the state before the step as densities, once for all its Newton iterations
          const Slots sl = slots_at(L, i);
          const size_t ob = (size_t)i * 4 * Bp + l;
          a.BD[ob] = exp(*W.y(bk, i, 1));
          a.BD[ob + Bp] = exp(*W.y(bk, i, 2));
          a.BD[ob + 2 * Bp] = sl.a >= 0 ? exp(*W.y(bk, i, 3)) : 0.0;
          a.BD[ob + 3 * Bp] = sl.c >= 0 ? exp(*W.y(bk, i, 4)) : 0.0;
          V = *W.y(bn, i, 0);
        } else {
          V = L.VL() - 0.5 * L.left() * Vi;
        }
        if (!(dti > 0.0)) {
          const Slots sl = slots_at(L, i);
          const double hL = L.st(i - 1, S_H) * L.L;
          // anions exp(+V/V_T), cations exp(-V/V_T) (their steady rows, `_ion_logs`)
          if (sl.a >= 0 && sl.a == slp.a)
            num[sl.a] += 0.5 * (exp(Vprev * L.iVt) + exp(V * L.iVt)) * hL;
          if (sl.c >= 0 && sl.c == slp.c)
            num[L.ka + sl.c] += 0.5 * (exp(-Vprev * L.iVt) + exp(-V * L.iVt)) * hL;
          slp = sl;
        }
        Vprev = V;
      }
    }
    if constexpr (TW) {  // both halves' numbers, added in one order; the points in memory
#pragma unroll
      for (int q = 0; q < K; ++q) num[q] = psum(mask, top, num[q]);
      __syncwarp(mask);
    }
    double lg[K];
#pragma unroll
    for (int q = 0; q < K; ++q) {
      if (dti > 0.0) {
        lg[q] = moving ? logs[q] + clipd(rt * (logs[q] - logs_p[q]), -ION_LOG_CAP, ION_LOG_CAP)
                       : 0.0;
      } else {
        lg[q] = L.tot[q] > 0.0 ? log(L.tot[q] / num[q]) : 0.0;
      }
    }
    // ---- Newton (batch._newton_loop, batch.py:740-848)
    double sh[STALL_STEPS + 1], jh[STALL_STEPS + 1];
#pragma unroll
    for (int q = 0; q <= STALL_STEPS; ++q) { sh[q] = INFINITY; jh[q] = INFINITY; }
    int it = 0;
    bool done = false, finite = true;
    while (!done && it < a.max_iter && !isnan(sh[STALL_STEPS])) {
      finite = true;  // of this iteration's new iterate
      double size = 0.0;
      if constexpr (TW) {
        tw_iteration<K>(a, W, bn, Vi, dti, lg, top, mask, capV, size, finite);
      } else {
      // -------- assembly and forward elimination
      double cpv[5][5], dpv[5][NC];
#pragma unroll
      for (int r = 0; r < 5; ++r) {
#pragma unroll
        for (int c = 0; c < 5; ++c) cpv[r][c] = 0.0;
#pragma unroll
        for (int c = 0; c < NC; ++c) dpv[r][c] = 0.0;
      }
      double gnum[K];
#pragma unroll
      for (int q = 0; q < K; ++q) gnum[q] = 0.0;
      TP pm, pc, pn;
      load_point(W, bn, 0, Vi, pm);
      contact_ions(W, bn, 0, dti, pm);
      load_point(W, bn, 1, Vi, pc);
      Flux el, er;
      flux(L, pm.c, pc.c, L.st(0, S_MUN), L.st(0, S_MUP), el);
      double elg[K];  // the slots' scales, once per iteration
#pragma unroll
      for (int q = 0; q < K; ++q) elg[q] = exp(lg[q]);
      IonIv ivl[2], ivr[2];  // the ions' fluxes of the row's left and right intervals
      ion_ivs(W, 0, pm, pc, ivl);
      for (int i = 1; i <= NP; ++i) {
        load_point(W, bn, i + 1, Vi, pn);
        contact_ions(W, bn, i + 1, dti, pn);
        flux(L, pc.c, pn.c, L.st(i, S_MUN), L.st(i, S_MUP), er);
        ion_ivs(W, i, pc, pn, ivr);
        const double hm = L.st(i - 1, S_H), hp = L.st(i, S_H);
        const int ifm = (int)L.st(i - 1, S_IFK), ifi = (int)L.st(i, S_IFK);
        const double fb = FB[(size_t)i * Bp + l];
        const double fim = ifm >= 0 ? FI[(size_t)(i - 1) * Bp + l] : 0.0;
        const double fii = ifi >= 0 ? FI[(size_t)i * Bp + l] : 0.0;
        const size_t ob = (size_t)i * 4 * Bp + l;
        const double bnv = a.BD[ob], bpv = a.BD[ob + Bp];
        const double bav = a.BD[ob + 2 * Bp], bcv = a.BD[ob + 3 * Bp];
        double A[5][5], Bm[5][5], Cm[5][5], r[5], U[5][K];
        row5<K>(W, i, pm, pc, pn, el, er, hm, hp, ifm, ifi, dti, fb, fim, fii, bnv, bpv, bav, bcv,
                lg, A, Bm, Cm, r, U, nullptr, nullptr, elg, ivl, ivr);
        // with VINT the rows' derivatives in the internal voltage, through the contacts'
        // potentials V0 + left Vint / 2 and VL - left Vint / 2 (`_system_vint`'s column)
        double uv[5];
#pragma unroll
        for (int rr = 0; rr < 5; ++rr)
          uv[rr] = VINT ? (i == 1 ? A[rr][0] * 0.5 * L.left() : 0.0) +
                              (i == NP ? Cm[rr][0] * (-0.5 * L.left()) : 0.0)
                        : 0.0;
        ivl[0] = ivr[0];
        ivl[1] = ivr[1];
        // the ions' numbers over interval i-1 (between points i-1 and i)
        {
          const double hL = hm * L.L;
          if (pc.c.sl.a >= 0 && pc.c.sl.a == pm.c.sl.a)
            gnum[pc.c.sl.a] += 0.5 * (pm.a + pc.a) * hL;
          if (pc.c.sl.c >= 0 && pc.c.sl.c == pm.c.sl.c)
            gnum[L.ka + pc.c.sl.c] += 0.5 * (pm.c2 + pc.c2) * hL;
        }
        // M = B - A c'_{i-1}; right-hand sides [C | -F | U] - A [0 | d'_{i-1}]
        double M[5][5];
#pragma unroll
        for (int rr = 0; rr < 5; ++rr)
#pragma unroll
          for (int c = 0; c < 5; ++c) {
            double s = Bm[rr][c];
#pragma unroll
            for (int q = 0; q < 5; ++q) s -= A[rr][q] * cpv[q][c];
            M[rr][c] = s;
          }
        double rhs[5][NC];
#pragma unroll
        for (int rr = 0; rr < 5; ++rr) {
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            double s = c == 0 ? r[rr] : (VINT && c == NC - 1) ? uv[rr] : U[rr][c - 1];
#pragma unroll
            for (int q = 0; q < 5; ++q) s -= A[rr][q] * dpv[q][c];
            rhs[rr][c] = s;
          }
        }
        Part f;
        partition(M, f);
#pragma unroll
        for (int c = 0; c < 5; ++c) {
          double v[5] = {Cm[0][c], Cm[1][c], Cm[2][c], Cm[3][c], Cm[4][c]};
          apply(f, v);
#pragma unroll
          for (int rr = 0; rr < 5; ++rr) { cpv[rr][c] = v[rr]; *cd(i, rr * 5 + c) = v[rr]; }
        }
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          double v[5] = {rhs[0][c], rhs[1][c], rhs[2][c], rhs[3][c], rhs[4][c]};
          apply(f, v);
#pragma unroll
          for (int rr = 0; rr < 5; ++rr) { dpv[rr][c] = v[rr]; *cd(i, 25 + rr * NC + c) = v[rr]; }
        }
        pm = pc;
        pc = pn;
        el = er;
      }
      // the ions' numbers over the last interval, where a region reaches the right contact
      {
        const double hL = L.st(NP, S_H) * L.L;
        if (pc.c.sl.a >= 0 && pc.c.sl.a == pm.c.sl.a) gnum[pc.c.sl.a] += 0.5 * (pm.a + pc.a) * hL;
        if (pc.c.sl.c >= 0 && pc.c.sl.c == pm.c.sl.c)
          gnum[L.ka + pc.c.sl.c] += 0.5 * (pm.c2 + pc.c2) * hL;
      }
      // -------- back substitution with the slots' Schur complement
      double SM[KV][KV], sr[KV];
#pragma unroll
      for (int q = 0; q < KV; ++q) {
        const bool has = q < K && L.tot[q] > 0.0;
#pragma unroll
        for (int q2 = 0; q2 < KV; ++q2) SM[q][q2] = (q == q2 && !has) ? 1.0 : 0.0;
        sr[q] = q < K ? -(has ? gnum[q] / L.tot[q] - 1.0 : lg[q]) : 0.0;
      }
      {
        double xn[5][NC];
#pragma unroll
        for (int rr = 0; rr < 5; ++rr)
#pragma unroll
          for (int c = 0; c < NC; ++c) xn[rr][c] = 0.0;
        Slots s_next = slots_at(L, NP + 1), s_here = slots_at(L, NP);
        for (int i = NP; i >= 1; --i) {
          double xi[5][NC];
#pragma unroll
          for (int rr = 0; rr < 5; ++rr)
#pragma unroll
            for (int c = 0; c < NC; ++c) {
              double s = *cd(i, 25 + rr * NC + c);
#pragma unroll
              for (int q = 0; q < 5; ++q) s -= *cd(i, rr * 5 + q) * xn[q][c];
              xi[rr][c] = s;
            }
#pragma unroll
          for (int rr = 0; rr < 5; ++rr)
#pragma unroll
            for (int c = 0; c < NC; ++c) {
              *cd(i, 25 + rr * NC + c) = xi[rr][c];
              xn[rr][c] = xi[rr][c];
            }
          // the constraints' border: W = d g / d (ln a_i or ln c_i)
          const Slots s_prev = slots_at(L, i - 1);
          const double hLm = L.st(i - 1, S_H) * L.L, hLp = L.st(i, S_H) * L.L;
#pragma unroll
          for (int sp = 0; sp < 2; ++sp) {
            const int sl = sp == 0 ? s_here.a : s_here.c;
            if (sl < 0) continue;
            const int q = sp == 0 ? sl : L.ka + sl;
            if (!(L.tot[q] > 0.0)) continue;
            const int slm = sp == 0 ? s_prev.a : s_prev.c, sln = sp == 0 ? s_next.a : s_next.c;
            const double wpt = 0.5 * ((slm == sl ? hLm : 0.0) + (sln == sl ? hLp : 0.0));
            double w = wpt * exp(*W.y(bn, i, 3 + sp)) / L.tot[q], wv = 0.0;
            // a region that reaches a contact: the contact's density follows this point's
            if ((i == 1 && slm == sl) || (i == NP && sln == sl)) {
              const int kc = i == 1 ? 0 : NP + 1;
              TP P;
              load_point(W, bn, kc, Vi, P);
              double dr;
              contact_ions(W, bn, kc, dti, P, &dr);
              const double wc = 0.5 * (i == 1 ? hLm : hLp) * (sp == 0 ? P.a : P.c2) / L.tot[q];
              w += wc;
              wv = wc * (sp == 0 ? dr : -dr);
            }
            sr[q] -= w * xi[3 + sp][0] + wv * xi[0][0];
#pragma unroll
            for (int q2 = 0; q2 < KV; ++q2)
              SM[q][q2] -= w * xi[3 + sp][1 + q2] + wv * xi[0][1 + q2];
          }
          s_next = s_here;
          s_here = s_prev;
        }
      }
      if constexpr (VINT)
        vint_row<K, NC>(a, W, bn, bk, Vi, V_k, V_now, dti, dti_now, oc_k, SM[K], sr[K]);
      double z[KV];
      small_solve<KV>(SM, sr, z);
      // -------- the damped update (batch.py:759-785)
      double dl_max = 0.0;
#pragma unroll
      for (int q = 0; q < K; ++q) {
        const double dlq = clipd(z[q], -ION_LOG_CAP, ION_LOG_CAP);
        dl_max = nanmax(dl_max, fabs(dlq));
        lg[q] += dlq;
      }
      if constexpr (VINT) {  // the voltage's step held to the potential's cap
        const double dV = clipd(z[K], -capV, capV);
        dl_max = nanmax(dl_max, fabs(dV) * L.iVt);
        Vi += dV;
      }
      for (int i = 1; i <= NP; ++i) {
        double d5[5];
#pragma unroll
        for (int rr = 0; rr < 5; ++rr) {
          double s = *cd(i, 25 + rr * NC);
#pragma unroll
          for (int q = 0; q < KV; ++q) s -= *cd(i, 25 + rr * NC + 1 + q) * z[q];
          d5[rr] = s;
        }
        double y5[5];
#pragma unroll
        for (int c = 0; c < 5; ++c) y5[c] = *W.y(bn, i, c);
        double st5[5];
        st5[0] = clipd(d5[0], -capV, capV);
#pragma unroll
        for (int c = 1; c < 5; ++c) st5[c] = clipd(d5[c], -CAP_LN, CAP_LN);
#pragma unroll
        for (int c = 1; c < 3; ++c) {  // a density below the floor steps in the density
          if (y5[c] < L.lognf) {
            const double dd = d5[c];
            const double in_n = dd > -1.0 ? log1p(dd) : -CAP_LN;
            st5[c] = clipd(in_n, -FLOOR_DROP_CAP, CAP_LN);
          }
        }
        size = nanmax(size, fabs(st5[0]) * L.iVt);
#pragma unroll
        for (int c = 0; c < 5; ++c) {
          const double nw = y5[c] + st5[c];
          *W.y(bn, i, c) = nw;
          finite = finite && isfinite(nw);
          if (c >= 1) {
            const double dens = exp(nw);
            size = nanmax(size, fabs(st5[c]) * (dens / (dens + L.nfloor)));
          }
        }
      }
      size = nanmax(size, dl_max);
#pragma unroll
      for (int q = 0; q < K; ++q) finite = finite && isfinite(lg[q]);
      }
      // -------- the current at the new iterate (half 0's, to both) and the stops
      double J = 0.0;
      J = current_t<K, false, TW>(W, bn, Vi, bk, V_now, dti, dti_now, FB, FI, nullptr, nullptr,
                                  top, mask);
#pragma unroll
      for (int q = 0; q < STALL_STEPS; ++q) { sh[q] = sh[q + 1]; jh[q] = jh[q + 1]; }
      sh[STALL_STEPS] = size;
      jh[STALL_STEPS] = J;
      ++it;
      double smax = sh[0], smin1 = sh[1], jdev = 0.0;
#pragma unroll
      for (int q = 1; q <= STALL_STEPS; ++q) smax = nanmax(smax, sh[q]);
#pragma unroll
      for (int q = 2; q <= STALL_STEPS; ++q) smin1 = fmin(smin1, sh[q]);
#pragma unroll
      for (int q = 0; q <= STALL_STEPS; ++q) jdev = nanmax(jdev, fabs(jh[q] - J));
      const bool stalled = it > STALL_STEPS && smax < ROUND_OFF_FLOOR && smin1 >= 0.1 * sh[0];
      const bool settled = !VINT && it > STALL_STEPS && size < CURRENT_STEP_CAP &&
                           jdev < CURRENT_TOL * (L.Jscale() + fabs(J));
      const bool quad = it > 1 && size < QUADRATIC_TOL &&
                        size < QUADRATIC_RATIO * sh[STALL_STEPS - 1];
      done = size < a.tol || stalled || settled || quad;
    }
    const bool ok = done;
    const double J = jh[STALL_STEPS];
    const double J_ext = J + L.Gshunt() * Vi;
    if (a.prof_state && top) write_profile(a, W, bn, k, Vi, dti);
    double err_k = 0.0;  // the step's errJ, where its convVar compares currents
    if ((a.COL || cv != 1) && top)
      columns_t<K>(a, W, bn, Vi, bk, V_now, dti, dti_now, J, J_ext, k, cv != 1 ? &err_k : nullptr);
    if constexpr (TW) err_k = __shfl_sync(mask, err_k, threadIdx.x & 30u);
    // ---- ZimT's main loop (transient.py:419-445)
    const bool running = stop == 0;
    const bool failed = running && !ok && (fm == 0 || (fm == 2 && track_curr == 1));
    const bool keep = running && !failed && finite && (ok || fm == 1 || (fm == 2 && dti == 0.0));
    if (keep) {
      // the tangents of this step, before the occupations move on (they take the old ones)
      const double dt = dti > 0.0 ? t_k - t_last : 0.0;
      Qint += J * dt;
      if (grad) tangent_step<K, VINT>(a, W, bn, bk, Vi, V_now, dti, dti_now, dt, lg, tb, dQ, tVv, oc_k);
      // the traps' occupations at the step's end, from its solution (and their tangents)
      auto tyn = [&](int p, int k, int c) {
        return (k < 1 || k > NP) ? 0.0
                                 : a.TY[((((size_t)(p * 2 + 1 - tb)) * tnodes + k) * 5 + c) * Bp + l];
      };
      // the traps' occupations at the step's end: with TW half 0 intervals 0 .. m - 1 (points
      // 1 .. m), half 1 the rest, after half 0's reads of the old ones (profile, columns)
      if constexpr (TW) __syncwarp(mask);
      const int mh = NP / 2;
      const int e_lo = TW && !top ? mh : 0, e_hi = TW && top ? mh - 1 : NP;
      TP pa, pb;
      load_point(W, bn, e_lo, Vi, pa);
      for (int e = e_lo; e <= e_hi; ++e) {
        load_point(W, bn, e + 1, Vi, pb);
        const int ifk = (int)L.st(e, S_IFK);
        if (ifk >= 0) {
          Iface t;
          double end;
          const double f_old = FI[(size_t)e * Bp + l];
          iface_edge_t(L, ifk, pa.c.n, pb.c.n, pa.c.p, pb.c.p, f_old, dti, t, false, &end);
          FI[(size_t)e * Bp + l] = end;
          if (grad && L.itab(ifk, I_NT) > 0.0) {
            TrapStep o;
            trap_step(L.itab(ifk, I_CN), L.itab(ifk, I_CP),
                      L.itab(ifk, I_NT0LO) + L.itab(ifk, I_NT0HI),
                      L.itab(ifk, I_PT0LO) + L.itab(ifk, I_PT0HI), pa.c.n + pb.c.n,
                      pa.c.p + pb.c.p, f_old, dti, o);
#pragma unroll
            for (int p = 0; p < 2; ++p) {
              double& tf = a.TFI[((size_t)p * tnodes + e) * Bp + l];
              tf = o.Ef * tf + o.en * (pa.c.n * tyn(p, e, 1) + pb.c.n * tyn(p, e + 1, 1)) +
                   o.ep * (pa.c.p * tyn(p, e, 2) + pb.c.p * tyn(p, e + 1, 2));
            }
          }
        }
        if (e + 1 <= NP && L.st(e + 1, S_NT) > 0.0) {
          const size_t o = (size_t)(e + 1) * Bp + l;
          if (grad) {
            TrapStep ts_;
            trap_step(L.st(e + 1, S_CNT), L.st(e + 1, S_CPT), L.st(e + 1, S_NT0),
                      L.st(e + 1, S_PT0), pb.c.n, pb.c.p, FB[o], dti, ts_);
#pragma unroll
            for (int p = 0; p < 2; ++p) {
              double& tf = a.TFB[((size_t)p * tnodes + e + 1) * Bp + l];
              tf = ts_.Ef * tf + ts_.en * pb.c.n * tyn(p, e + 1, 1) +
                   ts_.ep * pb.c.p * tyn(p, e + 1, 2);
            }
          }
          FB[o] = bulk_end(L, e + 1, pb.c.n, pb.c.p, FB[o], dti);
        }
        pa = pb;
      }
      const int old_p = bp;
      bp = bk; bk = bn; bn = old_p;
      tb = 1 - tb;
#pragma unroll
      for (int q = 0; q < K; ++q) { logs_p[q] = logs[q]; logs[q] = lg[q]; }
      V_before = V_now;
      V_now = Vi;
      J_ext_now = J_ext;
      dti_now = dti;
      track_curr = a.track[so];
      t_last = t_k;
      G_cur = L.gfrac;
      J_cur = J;
      err_cur = err_k;
    }
    // ZimT's automatic stop by the last state kept (transient.py:432-442): Track 1 makes it the
    // reference where the step converged; 2 and 3 count equal states in a row (where the step
    // converged or failureMode is 1), 3 then makes it the reference
    const bool counted = running && !failed && (track_curr == 2 || track_curr == 3) &&
                         (ok || fm == 1);
    if (counted)
      count = (a.tolp && a.told && G_ref == G_cur &&
               states_equal(a, W, bk, V_now, dti_now, cv, J_ref - J_cur, fmin(err_ref, err_cur)))
                  ? count + 1
                  : 0;
    const bool becomes_ref = running && !failed &&
                             ((track_curr == 1 && ok) || (track_curr == 3 && (ok || fm == 1)));
    if (becomes_ref && a.REF) {
      if (top) write_ref(a, W, bk, V_now, dti_now);
      G_ref = G_cur;
      J_ref = J_cur;
      err_ref = err_cur;
    }
    if (failed) stop = STOP_FAILED;
    else if (running && count >= MIN_COUNT_STATIC) stop = STOP_STATIC;
    first = false;
    const size_t o = (size_t)k * Bp + l;
    if (top) {
      a.J[o] = J;
      a.Jext[o] = J_ext;
      a.conv[o] = ok ? 1 : 0;
      a.iters[o] = it;
      a.acc[o] = keep ? 1 : 0;
      if (a.Vout) a.Vout[o] = Vi;
    }
  }
  if (!top) return;  // the outputs below are half 0's
  a.stop[l] = stop;
  if (grad) {
    a.Qout[l] = Qint;
    a.dQout[l] = dQ[0];
    a.dQout[(size_t)Bp + l] = dQ[1];
  }
  for (int i = 0; i <= NP + 1; ++i) {
    TP p;
    load_point(W, bk, i, V_now, p);
    contact_ions(W, bk, i, dti_now, p);
    const double v5[5] = {p.c.V, p.c.lnn, p.c.lnp, p.la, p.lc};
#pragma unroll
    for (int c = 0; c < 5; ++c) a.state_out[((size_t)i * 5 + c) * Bp + l] = v5[c];
  }
#pragma unroll
  for (int q = 0; q < K; ++q) a.logs_out[(size_t)q * Bp + l] = logs[q];
  for (int i = 0; i <= NP + 1; ++i) {
    const size_t o = (size_t)i * Bp + l;
    if (a.fb_out) a.fb_out[o] = (i >= 1 && i <= NP) ? FB[o] : 0.0;
    if (a.fi_out) a.fi_out[o] = i <= NP ? FI[o] : 0.0;
  }
}

}  // namespace tr
}  // namespace dd

// ------------------------------------------------------------------------------------ C ABI

namespace {

int slots_k_t(const dd_batch* b) { return b->k_anion + b->k_cation <= 2 ? 2 : 4; }

size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

void ws_parts(const dd_batch* b, size_t* y, size_t* fb, size_t* fi, size_t* cd, int* ncd,
              size_t* tan) {
  const int K = slots_k_t(b);
  const size_t nodes = (size_t)b->np_max + 2, Bp = (size_t)b->lane_stride;
  // the Newton step's 1 + K columns (2 + K with the internal voltage an unknown), or the
  // tangents' 2 + K (3 + K)
  *ncd = 25 + 5 * (3 + K);
  *y = align_up(3 * nodes * 5 * Bp * sizeof(double));
  *fb = align_up(nodes * Bp * sizeof(double));
  *fi = align_up(nodes * Bp * sizeof(double));
  *cd = align_up(nodes * (size_t)(*ncd) * Bp * sizeof(double))
        + align_up(nodes * 4 * Bp * sizeof(double));  // and the before-state record
  // the tangents: two parameters' states (two buffers each) and traps' occupations
  *tan = align_up(4 * nodes * 5 * Bp * sizeof(double)) + 2 * align_up(2 * nodes * Bp * sizeof(double));
  // and the automatic stop's reference state
  *tan += align_up(nodes * 5 * Bp * sizeof(double));
}

bool batch_ok(const dd_batch* b) {
  return b && b->n_lanes >= 1 && b->lane_stride >= b->n_lanes && b->np_max >= 1 &&
         b->k_anion >= 1 && b->k_cation >= 1 && b->k_anion + b->k_cation <= dd::DD_MAXK;
}

}  // namespace

extern "C" {

int dd_transient_workspace_bytes(const dd_batch* batch, size_t* bytes) {
  if (!batch_ok(batch) || !bytes) return DD_ERR_ARGS;
  size_t y, fb, fi, cd, tan;
  int ncd;
  ws_parts(batch, &y, &fb, &fi, &cd, &ncd, &tan);
  *bytes = y + fb + fi + cd + tan;
  return DD_OK;
}

int dd_transient(const dd_batch* batch, const double* tstat, const dd_steps* steps,
                 const double* start, const double* start_logs, const dd_transient_init* initial,
                 const dd_opts* opts, const dd_transient_out* out, void* workspace,
                 size_t workspace_bytes, void* stream) {
  if (!batch_ok(batch) || !batch->stat || !batch->scal || !batch->iface || !tstat || !steps ||
      !opts || !out || !workspace)
    return DD_ERR_ARGS;
  if (initial ? (!initial->state || !initial->f_bulk || !initial->f_iface || !initial->scalars)
              : (!start || !start_logs))
    return DD_ERR_ARGS;
  const bool prof = out->prof_state || out->prof_f_bulk || out->prof_f_iface || out->prof_dti;
  if (prof && !(out->prof_state && out->prof_f_bulk && out->prof_f_iface && out->prof_dti))
    return DD_ERR_ARGS;
  if (steps->n_steps < 1 || !steps->t || !steps->v || !steps->g_frac || !steps->track ||
      !steps->failure_mode || (steps->stride != 0 && steps->stride != batch->lane_stride))
    return DD_ERR_ARGS;
  if (steps->vint && (!steps->oc || !steps->r_series || !steps->start_j_ext)) return DD_ERR_ARGS;
  // The internal voltage an unknown with an ion region that reaches a contact (the transient
  // and its gradients) is not built: the host (jaxdd_b200/transient.py) refuses it before any
  // launch; this entry point does not check it.
  if (!out->J || !out->J_ext || !out->converged || !out->iterations || !out->accepted ||
      !out->stop || !out->state || !out->logs)
    return DD_ERR_ARGS;
  if (opts->max_iter < 1 || !(opts->tol > 0.0)) return DD_ERR_ARGS;
  size_t y, fb, fi, cd, tan;
  int ncd;
  ws_parts(batch, &y, &fb, &fi, &cd, &ncd, &tan);
  if (workspace_bytes < y + fb + fi + cd + tan) return DD_ERR_WORKSPACE;
  if ((out->Q == nullptr) != (out->dQ == nullptr)) return DD_ERR_ARGS;
  char* w = static_cast<char*>(workspace);
  dd::tr::Args a;
  a.S = batch->stat; a.C = batch->scal; a.IFt = batch->iface; a.X = tstat;
  a.n = batch->n_lanes; a.Bp = batch->lane_stride; a.npmax = batch->np_max;
  a.ka = batch->k_anion; a.kc = batch->k_cation;
  a.steps = steps->n_steps; a.tstride = steps->stride;
  a.t = steps->t; a.V = steps->v; a.G = steps->g_frac; a.track = steps->track;
  a.fmode = steps->failure_mode;
  a.y0 = start; a.logs0 = start_logs;
  a.tol = opts->tol; a.max_iter = opts->max_iter;
  a.simss = opts->bernoulli == DD_BERNOULLI_SIMSS;
  a.zimt = steps->zimt_sums != 0;
  a.ion_last = steps->zimt_ion_last != 0;
  a.Yb = reinterpret_cast<double*>(w);
  a.FB = reinterpret_cast<double*>(w + y);
  a.FI = reinterpret_cast<double*>(w + y + fb);
  a.CD = reinterpret_cast<double*>(w + y + fb + fi);
  a.ncd = ncd;
  a.BD = a.CD + ((size_t)batch->np_max + 2) * ncd * batch->lane_stride;
  a.J = out->J; a.Jext = out->J_ext; a.conv = out->converged; a.iters = out->iterations;
  a.acc = out->accepted; a.stop = out->stop; a.state_out = out->state; a.logs_out = out->logs;
  a.fb_out = out->f_bulk; a.fi_out = out->f_iface;
  a.Qout = out->Q; a.dQout = out->dQ;
  a.prof_state = out->prof_state; a.prof_fb = out->prof_f_bulk; a.prof_fi = out->prof_f_iface;
  a.prof_dti = out->prof_dti;
  a.init_state = initial ? initial->state : nullptr;
  a.init_fb = initial ? initial->f_bulk : nullptr;
  a.init_fi = initial ? initial->f_iface : nullptr;
  a.init_scal = initial ? initial->scalars : nullptr;
  a.oc = steps->oc; a.rser = steps->r_series; a.jext0 = steps->start_j_ext;
  a.Vout = out->V_int;
  a.tolp = steps->tol_pois; a.told = steps->tol_dens;
  a.convv = steps->conv_var; a.tolc = steps->tol_curr;
  a.LAY = steps->layers; a.nlay = steps->n_layers; a.COL = out->columns;
  if (a.COL && (!a.LAY || a.nlay < 1 || a.nlay > dd::tr::COL_MAXL)) return DD_ERR_ARGS;
  {
    const size_t nodes = (size_t)batch->np_max + 2, Bp = batch->lane_stride;
    a.REF = reinterpret_cast<double*>(w + y + fb + fi + cd + tan) -
            nodes * 5 * Bp;  // the last part of the tangents' region
  }
  if (out->Q) {
    const size_t nodes = (size_t)batch->np_max + 2, Bp = batch->lane_stride;
    char* t = w + y + fb + fi + cd;
    a.TY = reinterpret_cast<double*>(t);
    a.TFB = reinterpret_cast<double*>(t + align_up(4 * nodes * 5 * Bp * sizeof(double)));
    a.TFI = reinterpret_cast<double*>(t + align_up(4 * nodes * 5 * Bp * sizeof(double)) +
                                      align_up(2 * nodes * Bp * sizeof(double)));
  } else {
    a.TY = nullptr; a.TFB = nullptr; a.TFI = nullptr;
  }
  const int dst = dd::device_status();
  if (dst != DD_OK) return dst;
  const dim3 grid((batch->n_lanes + 31) / 32), block(32);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool k2 = slots_k_t(batch) == 2;
  if (steps->vint)
    return k2 ? dd::launch(dd::tr::transient_kernel<2, true>, grid, block, 0, s, a)
              : dd::launch(dd::tr::transient_kernel<4, true>, grid, block, 0, s, a);
  if (out->Q)  // the gradients: one thread a device
    return k2 ? dd::launch(dd::tr::transient_kernel<2, false>, grid, block, 0, s, a)
              : dd::launch(dd::tr::transient_kernel<4, false>, grid, block, 0, s, a);
  // two threads a device: the twisted sweep
  const dim3 grid2((2 * batch->n_lanes + 31) / 32);
  return k2 ? dd::launch(dd::tr::transient_kernel<2, false, true>, grid2, block, 0, s, a)
            : dd::launch(dd::tr::transient_kernel<4, false, true>, grid2, block, 0, s, a);
}

}  // extern "C"
