// Batched steady-state drift-diffusion J-V solve for sm_100a: one persistent launch, one thread
// per device ("lane"), every array lane-interleaved (dd_layout.h).
//
// What it computes is jaxdd's solve_batch / solve_jv (src/jaxdd/batch.py, src/jaxdd/solver.py):
// Newton on (V, ln n, ln p) at every interior point, the residual and 3x3 Jacobian blocks of
// SIMsalabim's Scharfetter-Gummel discretisation (`_assemble`, solver.py:1021-1187), the block
// tridiagonal system bordered by the mobile ions' K normalisations (`_bordered_solve`,
// batch.py:595-603), SIMsalabim's integral current (`_current`, batch.py:302-403), the damped
// Newton loop and its stops (`_newton_loop`, batch.py:740-848), the Poisson start and ion stages
// (`_start`, batch.py:875-934) and the outward voltage scan (`_solve_one`, batch.py:937-1006).
//
// How it computes it is this file's own:
//  * A Newton step is two passes over the grid. The forward pass assembles row i in registers
//    (each interval's fluxes once, carried to the next row), eliminates it at once
//    (M = B - A c', c' = M^-1 C, d' = M^-1 (r - A d')), and writes only c' and d'. It also
//    carries w' = U^-T W (U the unit upper factor of the sweep, W the constraints' border), so
//    that W^T T^-1 [r | U] = sum w'^T d' is known when the forward pass ends: the K x K Schur
//    complement is solved before the backward pass, and one back substitution with the right
//    side d'_F - d'_U z gives the bordered step directly.
//  * The backward pass back-substitutes, damps (`density_steps`), updates the state in place,
//    measures the step, and accumulates the terminal current right to left (the integral form's
//    prefix sums rewritten as suffix sums), so the current needs no pass of its own.
//  * Each lane runs its own program (start, pre-bias, scan) as a state machine; every loop
//    iteration takes one Newton (or Poisson) step in every lane, at that lane's own voltage.
//    Lanes never wait for another lane's voltage, so jaxdd's two passes (first_max_iter, then
//    stragglers, batch.py:1194-1208) collapse into one pass at max_iter with the same results.
//  * Every loop is bounded (caps on Poisson and Newton steps, voltages, stages): the kernel
//    always terminates.
#include <cuda_runtime.h>
#include <stdint.h>

#include "dd_layout.h"
#include "../../include/jaxdd_b200.h"

namespace dd {

constexpr double Q = 1.6022e-19;
constexpr double ROUND_OFF_FLOOR = 1e-6;
constexpr int STALL_STEPS = 3;
constexpr double NOISE_FLOOR_CAP = 1e-3;
constexpr double CAP_V = 10.0;  // in V_T
constexpr double CAP_LN = 5.0;
constexpr double ION_LOG_CAP = 5.0;
constexpr double FLOOR_DROP_CAP = 50.0;
constexpr double CURRENT_TOL = 1e-5;
constexpr double CURRENT_STEP_CAP = 1e-3;
constexpr double QUADRATIC_TOL = 1e-5;
constexpr double QUADRATIC_RATIO = 1e-2;
constexpr double POISSON_TOL = 1e-8;
constexpr double EPS64 = 2.220446049250313e-16;

__device__ __constant__ double c_stage_share[4] = {1.0 / 64, 1.0 / 16, 1.0 / 4, 1.0};

// ------------------------------------------------------------------------------------ helpers

__device__ __forceinline__ double clipd(double x, double lo, double hi) {
  // NaN passes through, as jnp.clip does
  return x < lo ? lo : (x > hi ? hi : x);
}
__device__ __forceinline__ double nanmax(double a, double b) {
  // a NaN anywhere stays: the reference's jnp.max propagates it
  return (b > a || b != b) ? b : a;
}

// B(|x|) and B'(|x|) for |x| >= 0: the exact function (series below 1e-2, solver.py:95-105) or
// SIMsalabim's (Taylor of order 1, 2, 4 below 0.05, 0.45, 1.5; solver.py:108-121). B(-|x|) is
// then B(|x|) + |x| (the identity B(-x) = B(x) + x, exact for both), which needs no second
// expm1 and keeps both values accurate.
__device__ __forceinline__ void bern_abs(double a, int simss, double& b, double& db) {
  if (simss) {
    if (a < 0.05) { b = 1.0 - 0.5 * a; db = -0.5; return; }
    if (a < 0.45) { b = 1.0 - a * (0.5 - a / 12.0); db = -0.5 + a / 6.0; return; }
    if (a < 1.5) {
      b = 1.0 + a * (-0.5 + a * (1.0 / 12.0 - a * a / 720.0));
      db = -0.5 + a / 6.0 - a * a * a / 180.0;
      return;
    }
  } else if (a < 1e-2) {
    b = 1.0 - a / 2.0 + a * a / 12.0 - a * a * a * a / 720.0;
    db = -0.5 + a / 6.0 - a * a * a / 180.0;
    return;
  }
  const double e = expm1(a);
  b = a / e;
  db = (1.0 - b) / e - b;  // 1/e - a(e+1)/e^2, finite where e overflows
}

// B(x), B(-x) and their derivatives B'(x), B'(-x) (as functions of their own argument).
__device__ __forceinline__ void bern_pair(double x, int simss, double& bf, double& bb,
                                          double& dbf, double& dbb) {
  double b, db;
  const double a = fabs(x);
  bern_abs(a, simss, b, db);
  if (x >= 0.0) { bf = b; dbf = db; bb = b + a; dbb = -db - 1.0; }
  else { bb = b; dbb = db; bf = b + a; dbf = -db - 1.0; }
}

// ------------------------------------------------------------------------------------ lane

struct Lane {
  // batch
  const double* __restrict__ S;
  const double* __restrict__ C;
  const double* __restrict__ IFt;
  int Bp, l, NP, ka, K;
  double Vt, iVt, L, V0, VL, left, lnnL, lnpL, lnnR, lnpR, Jscale, Gshunt, gfrac, nfloor,
      lognf, Hsum;
  int currdiff, simss;
  double tot[DD_MAXK];
  // dynamic
  double* Y;    // state buffers base: [DD_NBUF][np+2][3][Bp]
  double* FX;   // frozen ion densities [np+2][2][Bp]
  double* CD;   // sweep scratch [np+2][ncd][Bp]
  int ncd;      // fields per node in CD
  size_t ybuf;  // elements per state buffer
  bool frozen;
  double share;

  __device__ __forceinline__ double st(int k, int f) const {
    return __ldg(S + ((size_t)k * DD_NF + f) * Bp + l);
  }
  __device__ __forceinline__ double sc(int f) const { return __ldg(C + (size_t)f * Bp + l); }
  __device__ __forceinline__ double itab(int row, int f) const {
    return __ldg(IFt + ((size_t)row * DD_NIF + f) * Bp + l);
  }
  __device__ __forceinline__ double* y(int buf, int k, int c) const {
    return Y + buf * ybuf + ((size_t)k * 3 + c) * Bp + l;
  }
  __device__ __forceinline__ double* cd(int k, int f) const {
    return CD + ((size_t)k * ncd + f) * Bp + l;
  }
  __device__ __forceinline__ double afix(int k) const {
    return frozen ? FX[((size_t)k * 2) * Bp + l] : share * st(k, S_AFIX);
  }
  __device__ __forceinline__ double cfix(int k) const {
    return frozen ? FX[((size_t)k * 2 + 1) * Bp + l] : share * st(k, S_CFIX);
  }
  __device__ __forceinline__ double total(int k) const { return frozen ? 0.0 : share * tot[k]; }
};

// Slot of a point for each species, -1 where the species is not mobile there (or frozen).
struct Slots {
  int a, c;
};

__device__ __forceinline__ Slots slots_at(const Lane& L, int k) {
  Slots s;
  s.a = (int)L.st(k, S_ASLOT);
  s.c = (int)L.st(k, S_CSLOT);
  if (L.frozen) { s.a = -1; s.c = -1; }
  return s;
}

// A grid point's state and what the rows need of it.
struct Pt {
  double V, lnn, lnp, n, p, offn, offp;
  Slots sl;
  double da, dc;  // mobile anion / cation density (Boltzmann in V, `_ion_densities`)
};

__device__ __forceinline__ void pt_fill(const Lane& L, Pt& P, int k, const double* logs) {
  P.n = exp(P.lnn);
  P.p = exp(P.lnp);
  P.offn = L.st(k, S_OFFN);
  P.offp = L.st(k, S_OFFP);
  P.sl = slots_at(L, k);
  P.da = P.sl.a >= 0 ? exp(logs[P.sl.a] + P.V * L.iVt) : 0.0;
  P.dc = P.sl.c >= 0 ? exp(logs[L.ka + P.sl.c] - P.V * L.iVt) : 0.0;
}

// The contacts' states (`_bounds`, batch.py:255-259).
__device__ __forceinline__ void contact(const Lane& L, int right, double Vint, Pt& P) {
  if (!right) { P.V = L.V0 + 0.5 * L.left * Vint; P.lnn = L.lnnL; P.lnp = L.lnpL; }
  else { P.V = L.VL - 0.5 * L.left * Vint; P.lnn = L.lnnR; P.lnp = L.lnpR; }
}

// One interval's Scharfetter-Gummel fluxes and their derivatives in its two points'
// (V, ln n, ln p) (`_assemble`, solver.py:1061-1082).
struct Flux {
  double Fn, n0V, n0n, n1V, n1n, Fp, p0V, p0p, p1V, p1p;
};

__device__ __forceinline__ void flux(const Lane& L, const Pt& a, const Pt& b, double mun,
                                     double mup, Flux& f) {
  const double cn = L.Vt * mun, cp = L.Vt * mup;
  const double xn = ((b.V + b.offn) - (a.V + a.offn)) * L.iVt;
  const double xp = ((b.V + b.offp) - (a.V + a.offp)) * L.iVt;
  double Bnf, Bnb, dBnf, dBnb, Bpf, Bpb, dBpf, dBpb;
  bern_pair(xn, L.simss, Bnf, Bnb, dBnf, dBnb);
  bern_pair(xp, L.simss, Bpf, Bpb, dBpf, dBpb);
  f.Fn = cn * (Bnf * b.n - Bnb * a.n);
  const double gn = cn * (dBnf * b.n + dBnb * a.n) * L.iVt;
  f.n0V = -gn; f.n0n = -cn * Bnb * a.n;
  f.n1V = gn;  f.n1n = cn * Bnf * b.n;
  f.Fp = cp * (Bpf * a.p - Bpb * b.p);
  const double gp = cp * (dBpf * a.p + dBpb * b.p) * L.iVt;
  f.p0V = -gp; f.p0p = cp * Bpf * a.p;
  f.p1V = gp;  f.p1p = -cp * Bpb * b.p;
}

// Direct + SRH recombination at a point, and n dR/dn, p dR/dp (solver.py:734-745).
__device__ __forceinline__ void recomb(const Lane& L, int k, double n, double p, double& R,
                                       double& dRn, double& dRp) {
  const double kd = L.st(k, S_KD), ni2 = L.st(k, S_NI2), Nt = L.st(k, S_NT);
  R = kd * (n * p - ni2);
  dRn = n * kd * p;
  dRp = p * kd * n;
  if (Nt > 0.0) {
    const double Cn = L.st(k, S_CNT), Cp = L.st(k, S_CPT);
    const double nt0 = L.st(k, S_NT0), pt0 = L.st(k, S_PT0);
    const double den = Cn * (n + nt0) + Cp * (p + pt0);
    const double kk = Nt * Cn * Cp;
    const double srh = kk * (n * p - nt0 * pt0) / den;
    R += srh;
    dRn += n * (kk * p - srh * Cn) / den;
    dRp += p * (kk * n - srh * Cp) / den;
  }
}

// Interface traps of one interval (table row t), steady state, one level (solver.py:814-850):
// v = (Rn_L, Rn_R, Rp_L, Rp_R, Q) and, when asked, their derivatives in ln nL, ln nR, ln pL, ln pR.
struct Iface {
  double v[5];
  double d[4][5];
};

__device__ void iface_edge(const Lane& L, int t, double nL, double nR, double pL, double pR,
                           Iface& o, bool derivs) {
  const double Nt = L.itab(t, I_NT), Cn = L.itab(t, I_CN), Cp = L.itab(t, I_CP);
  const double nlo = L.itab(t, I_NT0LO), nhi = L.itab(t, I_NT0HI);
  const double plo = L.itab(t, I_PT0LO), phi = L.itab(t, I_PT0HI);
  const double iw = L.itab(t, I_IW);
  const double hq = L.itab(t, I_CHARGE) * 0.5 * Nt * iw, cwe = L.itab(t, I_CWE);
  const double an = Cn * Nt, bp = Cp * Nt;
  const double a = an * (nL + nR), b = bp * (pL + pR), c = an * (nlo + nhi), d = bp * (plo + phi);
  const double inv = Nt > 0.0 ? 1.0 / (a + b + c + d) : 0.0;
  const double full = (a + d) * inv, empty = (b + c) * inv;
  o.v[0] = iw * an * (nL * empty - nlo * full);
  o.v[1] = iw * an * (nR * empty - nhi * full);
  o.v[2] = iw * bp * (pL * full - plo * empty);
  o.v[3] = iw * bp * (pR * full - phi * empty);
  o.v[4] = hq * (cwe - full);
  if (!derivs) return;
#pragma unroll
  for (int w = 0; w < 4; ++w) {
    double df, de;
    if (w < 2) {
      const double da = an * (w == 0 ? nL : nR);
      df = da * empty * inv; de = -da * empty * inv;
    } else {
      const double db = bp * (w == 2 ? pL : pR);
      df = -db * full * inv; de = db * full * inv;
    }
    o.d[w][0] = iw * an * ((w == 0 ? nL * empty : 0.0) + nL * de - nlo * df);
    o.d[w][1] = iw * an * ((w == 1 ? nR * empty : 0.0) + nR * de - nhi * df);
    o.d[w][2] = iw * bp * ((w == 2 ? pL * full : 0.0) + pL * df - plo * de);
    o.d[w][3] = iw * bp * ((w == 3 ? pR * full : 0.0) + pR * df - phi * de);
    o.d[w][4] = -hq * df;
  }
}

// The ion slots' numbers over one interval (`_ion_number`, trapezoidal, solver.py:1241-1252).
template <int K>
__device__ __forceinline__ void ion_edge(const Lane& L, const Pt& a, const Pt& b, double hL,
                                         double* num) {
  if (a.sl.a >= 0 && a.sl.a == b.sl.a) num[a.sl.a] += 0.5 * (a.da + b.da) * hL;
  if (a.sl.c >= 0 && a.sl.c == b.sl.c) num[L.ka + a.sl.c] += 0.5 * (a.dc + b.dc) * hL;
}

// The constraints' derivative in a point's potential (the reference's jacrev of
// `_ion_constraints`): its two intervals' trapezoid weights times its density over V_T.
template <int K>
__device__ __forceinline__ void ion_w(const Lane& L, const Pt& pm, const Pt& pc, const Pt& pn,
                                      double hLm, double hLp, double* W) {
#pragma unroll
  for (int k = 0; k < K; ++k) W[k] = 0.0;
  if (pc.sl.a >= 0) {
    const int k = pc.sl.a;
    const double tk = L.total(k);
    if (tk > 0.0) {
      const double wpt = 0.5 * ((pm.sl.a == k ? hLm : 0.0) + (pn.sl.a == k ? hLp : 0.0));
      W[k] = wpt * pc.da * L.iVt / tk;
    }
  }
  if (pc.sl.c >= 0) {
    const int k = L.ka + pc.sl.c;
    const double tk = L.total(k);
    if (tk > 0.0) {
      const double wpt = 0.5 * ((pm.sl.c == pc.sl.c ? hLm : 0.0) + (pn.sl.c == pc.sl.c ? hLp : 0.0));
      W[k] = -wpt * pc.dc * L.iVt / tk;
    }
  }
}

// Solve the K x K system M z = r by Gaussian elimination with partial pivoting.
template <int K>
__device__ void small_solve(double (&M)[K][K], double (&r)[K], double (&z)[K]) {
#pragma unroll
  for (int c = 0; c < K; ++c) {
    int piv = c;
    double best = fabs(M[c][c]);
#pragma unroll
    for (int rr = c + 1; rr < K; ++rr)
      if (fabs(M[rr][c]) > best) { best = fabs(M[rr][c]); piv = rr; }
    if (piv != c) {
#pragma unroll
      for (int j = 0; j < K; ++j) { double t = M[c][j]; M[c][j] = M[piv][j]; M[piv][j] = t; }
      double t = r[c]; r[c] = r[piv]; r[piv] = t;
    }
    const double inv = 1.0 / M[c][c];
#pragma unroll
    for (int rr = c + 1; rr < K; ++rr) {
      const double f = M[rr][c] * inv;
#pragma unroll
      for (int j = c; j < K; ++j) M[rr][j] -= f * M[c][j];
      r[rr] -= f * r[c];
    }
  }
#pragma unroll
  for (int c = K - 1; c >= 0; --c) {
    double s = r[c];
#pragma unroll
    for (int j = c + 1; j < K; ++j) s -= M[c][j] * z[j];
    z[c] = s / M[c][c];
  }
}

// ------------------------------------------------------------------------------------ advance

// How the first forward pass of a voltage makes its start from the carried solutions
// (`_solve_one`'s scan body, batch.py:964-1004): buffers 0 iterate, 1 carry, 2 previous carry,
// 3 the pre-bias solution.
enum Adv { ADV_NONE = 0, ADV_KEEP, ADV_NOKEEP, ADV_TURN };

__device__ __forceinline__ void load_state(const Lane& L, int k, int adv, double ratio, Pt& P) {
  double s[3];
  if (adv == ADV_NONE) {
#pragma unroll
    for (int c = 0; c < 3; ++c) s[c] = *L.y(0, k, c);
  } else {
    const double cap[3] = {CAP_V * L.Vt, CAP_LN, CAP_LN};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double base, prev;
      if (adv == ADV_KEEP) {  // the last solve converged: it is the carry, the old carry before it
        base = *L.y(0, k, c);
        prev = *L.y(1, k, c);
        *L.y(2, k, c) = prev;
        *L.y(1, k, c) = base;
      } else if (adv == ADV_NOKEEP) {
        base = *L.y(1, k, c);
        prev = *L.y(2, k, c);
      } else {  // the scan turns: both carries the pre-bias solution, no extrapolation
        base = *L.y(3, k, c);
        prev = base;
        *L.y(1, k, c) = base;
        *L.y(2, k, c) = base;
      }
      s[c] = base + clipd(ratio * (base - prev), -cap[c], cap[c]);
      *L.y(0, k, c) = s[c];
    }
  }
  P.V = s[0]; P.lnn = s[1]; P.lnp = s[2];
}

// ------------------------------------------------------------------------------------ current
//
// The terminal current (`_current_parts`, batch.py:316-403, steady state) is accumulated right
// to left in the backward pass, over the new state. For each carrier (electrons sn = -1, holes
// sn = +1), with U_k = R_k + R_int,k - G_k g (0 on the contacts), q_k = exp(sn Vg_k / V_T)/mu_k,
// c_k = (dx_{k-1} + dx_k)/2 and the trapezoids a_k = dx_k (U_k + U_{k+1})/2:
//   single = sum_k c_k q_k,  double = sum_k c_k q_k int_u_k = A single - sum_k c_k q_k T_k,
// T_k = sum_{e>=k} a_e the suffix sums (A = T_0), so no prefix sum is needed; and
//   sum_e h_e J_e = qK H + sum_k b_k Hs_k - sum_{interfaces e} h_e (b_e - t_e),
// b_k = sn q L h_k U_k, Hs_k = sum_{e>=k} h_e, t_e the current through interval e's traps
// (an interface's J is the one before it plus t_e). The differential form sums each interval's
// Scharfetter-Gummel flux, an interface again taking the interval before it plus t_e.

// ------------------------------------------------------------------------------------ Newton step

struct StepOut {
  double size;
  double J;
  bool finite;
};

// One Newton step of lane L at Vint (or, with `noise`, the round-off step of
// `_noise_step`, solver.py:1728-1751, which leaves the state as it is).
template <int K>
__device__ StepOut newton_step(Lane& L, double Vint, double* logs, int adv, double ratio,
                               bool noise) {
  const int NP = L.NP;
  const double Vt = L.Vt, iVt = L.iVt;
  const double gfrac = L.gfrac;
  // ---------------------------------------------------------------- forward
  Pt pm, pc, pn;
  contact(L, 0, Vint, pm);
  pt_fill(L, pm, 0, logs);
  load_state(L, 1, adv, ratio, pc);
  pt_fill(L, pc, 1, logs);
  Flux el;
  double h_m = L.st(0, S_H);
  flux(L, pm, pc, L.st(0, S_MUN), L.st(0, S_MUP), el);
  double num[K];
#pragma unroll
  for (int k = 0; k < K; ++k) num[k] = 0.0;
  ion_edge<K>(L, pm, pc, h_m * L.L, num);
  int ifk_m = (int)L.st(0, S_IFK);

  double cp[9];
  double dF[3], dU[3][K], wp[3][K];
  double Sm[K][K], sv[K];
#pragma unroll
  for (int j = 0; j < 9; ++j) cp[j] = 0.0;
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    dF[r] = 0.0;
#pragma unroll
    for (int k = 0; k < K; ++k) { dU[r][k] = 0.0; wp[r][k] = 0.0; }
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    sv[k] = 0.0;
#pragma unroll
    for (int j = 0; j < K; ++j) Sm[k][j] = 0.0;
  }

  for (int i = 1; i <= NP; ++i) {
    // the next point
    if (i < NP) load_state(L, i + 1, adv, ratio, pn);
    else contact(L, 1, Vint, pn);
    pt_fill(L, pn, i + 1, logs);
    const double h_i = L.st(i, S_H);
    const int ifk_i = (int)L.st(i, S_IFK);
    Flux er;
    flux(L, pc, pn, L.st(i, S_MUN), L.st(i, S_MUP), er);
    ion_edge<K>(L, pc, pn, h_i * L.L, num);

    // row i
    const double facl = L.st(i, S_FACL), facm = L.st(i, S_FACM), facu = L.st(i, S_FACU);
    const double fac = L.st(i, S_FAC), sP = L.st(i, S_SP), sC = L.st(i, S_SC);
    const double hm = h_m, hp = h_i;
    double R, dRn, dRp;
    recomb(L, i, pc.n, pc.p, R, dRn, dRp);
    const double gen = L.st(i, S_G) * gfrac;
    double elec = hm * er.Fn - hp * el.Fn + fac * (gen - R);
    double hole = hp * el.Fp - hm * er.Fp + fac * (gen - R);
    double pois = facl * pm.V + facm * pc.V + facu * pn.V -
                  Q * (pc.n - pc.p + L.st(i, S_DOP) + L.afix(i) + pc.da - L.cfix(i) - pc.dc);
    double A[3][3], Bm[3][3], Cm[3][3];
    A[0][0] = facl * sP; A[0][1] = 0.0; A[0][2] = 0.0;
    A[1][0] = -hp * el.n0V * sC; A[1][1] = -hp * el.n0n * sC; A[1][2] = 0.0;
    A[2][0] = hp * el.p0V * sC;  A[2][1] = 0.0;               A[2][2] = hp * el.p0p * sC;
    Bm[0][0] = (facm - Q * (pc.da + pc.dc) * iVt) * sP;
    Bm[0][1] = -Q * pc.n * sP;
    Bm[0][2] = Q * pc.p * sP;
    Bm[1][0] = (-hp * el.n1V + hm * er.n0V) * sC;
    Bm[1][1] = (-hp * el.n1n + hm * er.n0n - fac * dRn) * sC;
    Bm[1][2] = (-fac * dRp) * sC;
    Bm[2][0] = (hp * el.p1V - hm * er.p0V) * sC;
    Bm[2][1] = (-fac * dRn) * sC;
    Bm[2][2] = (hp * el.p1p - hm * er.p0p - fac * dRp) * sC;
    Cm[0][0] = facu * sP; Cm[0][1] = 0.0; Cm[0][2] = 0.0;
    Cm[1][0] = hm * er.n1V * sC; Cm[1][1] = hm * er.n1n * sC; Cm[1][2] = 0.0;
    Cm[2][0] = -hm * er.p1V * sC; Cm[2][1] = 0.0; Cm[2][2] = -hm * er.p1p * sC;
    if (ifk_m >= 0 || ifk_i >= 0) {
      // interface traps on the left interval (this point its right end) and/or the right one
      const double sc3[3] = {Q * sP, -fac * sC, -fac * sC};
      double X[3] = {0.0, 0.0, 0.0};
      Iface t;
      if (ifk_m >= 0) {
        iface_edge(L, ifk_m, pm.n, pc.n, pm.p, pc.p, t, true);
        const int hi[3] = {4, 1, 3};
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          X[r] += t.v[hi[r]];
          Bm[r][1] += sc3[r] * t.d[1][hi[r]];
          Bm[r][2] += sc3[r] * t.d[3][hi[r]];
          A[r][1] += sc3[r] * t.d[0][hi[r]];
          A[r][2] += sc3[r] * t.d[2][hi[r]];
        }
      }
      if (ifk_i >= 0) {
        iface_edge(L, ifk_i, pc.n, pn.n, pc.p, pn.p, t, true);
        const int lo[3] = {4, 0, 2};
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          X[r] += t.v[lo[r]];
          Bm[r][1] += sc3[r] * t.d[0][lo[r]];
          Bm[r][2] += sc3[r] * t.d[2][lo[r]];
          Cm[r][1] += sc3[r] * t.d[1][lo[r]];
          Cm[r][2] += sc3[r] * t.d[3][lo[r]];
        }
      }
      pois += Q * X[0];
      elec -= fac * X[1];
      hole -= fac * X[2];
    }
    double rhs[3];
    double U0[K];
    double W[K];
    if (!noise) {
      rhs[0] = -pois * sP; rhs[1] = -elec * sC; rhs[2] = -hole * sC;
#pragma unroll
      for (int k = 0; k < K; ++k) U0[k] = 0.0;
      if (pc.sl.a >= 0) U0[pc.sl.a] = -Q * pc.da * sP;
      if (pc.sl.c >= 0) U0[L.ka + pc.sl.c] = Q * pc.dc * sP;
      ion_w<K>(L, pm, pc, pn, h_m * L.L, h_i * L.L, W);
    } else {
      // each row's round-off: eps sum |d row / d y| |y| over its three points
      const double ym[3] = {fabs(pm.V), fabs(pm.lnn), fabs(pm.lnp)};
      const double yc[3] = {fabs(pc.V), fabs(pc.lnn), fabs(pc.lnp)};
      const double yn[3] = {fabs(pn.V), fabs(pn.lnn), fabs(pn.lnp)};
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        double s = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c)
          s += fabs(A[r][c]) * ym[c] + fabs(Bm[r][c]) * yc[c] + fabs(Cm[r][c]) * yn[c];
        rhs[r] = EPS64 * s;
      }
#pragma unroll
      for (int k = 0; k < K; ++k) { U0[k] = 0.0; W[k] = 0.0; }
    }
    // elimination: M = B - A c'
    double M[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        M[r][c] = Bm[r][c] - (A[r][0] * cp[c] + A[r][1] * cp[3 + c] + A[r][2] * cp[6 + c]);
    const double co00 = M[1][1] * M[2][2] - M[1][2] * M[2][1];
    const double co01 = M[0][2] * M[2][1] - M[0][1] * M[2][2];
    const double co02 = M[0][1] * M[1][2] - M[0][2] * M[1][1];
    const double co10 = M[1][2] * M[2][0] - M[1][0] * M[2][2];
    const double co11 = M[0][0] * M[2][2] - M[0][2] * M[2][0];
    const double co12 = M[0][2] * M[1][0] - M[0][0] * M[1][2];
    const double co20 = M[1][0] * M[2][1] - M[1][1] * M[2][0];
    const double co21 = M[0][1] * M[2][0] - M[0][0] * M[2][1];
    const double co22 = M[0][0] * M[1][1] - M[0][1] * M[1][0];
    const double idet = 1.0 / (M[0][0] * co00 + M[0][1] * co10 + M[0][2] * co20);
    const double Mi[3][3] = {{co00 * idet, co01 * idet, co02 * idet},
                             {co10 * idet, co11 * idet, co12 * idet},
                             {co20 * idet, co21 * idet, co22 * idet}};
    // w' = W e_0 - c'^T w'  (the previous c')
    double wn[3][K];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int k = 0; k < K; ++k)
        wn[r][k] = (r == 0 ? W[k] : 0.0) -
                   (cp[0 + r] * wp[0][k] + cp[3 + r] * wp[1][k] + cp[6 + r] * wp[2][k]);
    // d' = M^-1 (rhs - A d')
    double tF[3], tU[3][K];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      tF[r] = rhs[r] - (A[r][0] * dF[0] + A[r][1] * dF[1] + A[r][2] * dF[2]);
#pragma unroll
      for (int k = 0; k < K; ++k)
        tU[r][k] = (r == 0 ? U0[k] : 0.0) -
                   (A[r][0] * dU[0][k] + A[r][1] * dU[1][k] + A[r][2] * dU[2][k]);
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      dF[r] = Mi[r][0] * tF[0] + Mi[r][1] * tF[1] + Mi[r][2] * tF[2];
#pragma unroll
      for (int k = 0; k < K; ++k) dU[r][k] = Mi[r][0] * tU[0][k] + Mi[r][1] * tU[1][k] + Mi[r][2] * tU[2][k];
    }
    // c' = M^-1 C
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        cp[r * 3 + c] = Mi[r][0] * Cm[0][c] + Mi[r][1] * Cm[1][c] + Mi[r][2] * Cm[2][c];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int k = 0; k < K; ++k) wp[r][k] = wn[r][k];
    // the border's sums: sum w'^T d'
#pragma unroll
    for (int k = 0; k < K; ++k) {
      sv[k] += wp[0][k] * dF[0] + wp[1][k] * dF[1] + wp[2][k] * dF[2];
#pragma unroll
      for (int j = 0; j < K; ++j)
        Sm[k][j] += wp[0][k] * dU[0][j] + wp[1][k] * dU[1][j] + wp[2][k] * dU[2][j];
    }
    // store c', d'
#pragma unroll
    for (int j = 0; j < 9; ++j) *L.cd(i, j) = cp[j];
#pragma unroll
    for (int r = 0; r < 3; ++r) *L.cd(i, 9 + r) = dF[r];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int k = 0; k < K; ++k) *L.cd(i, 12 + r * K + k) = dU[r][k];
    // shift
    pm = pc; pc = pn; el = er; h_m = h_i; ifk_m = ifk_i;
  }

  // ---------------------------------------------------------------- border (Schur)
  double z[K];
#pragma unroll
  for (int k = 0; k < K; ++k) z[k] = 0.0;
  if (!noise) {
    double Msch[K][K], rr[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const double tk = L.total(k);
      const bool has = tk > 0.0;
      const double g = has ? num[k] / tk - 1.0 : 0.0;
      const double Dk = has ? num[k] / tk : 1.0;  // d g / d log, or the held identity
#pragma unroll
      for (int j = 0; j < K; ++j) Msch[k][j] = (j == k ? Dk : 0.0) - Sm[k][j];
      rr[k] = -g - sv[k];
    }
    small_solve<K>(Msch, rr, z);
  }

  // ---------------------------------------------------------------- backward
  StepOut out;
  out.size = 0.0;
  out.finite = true;
  double dlogs[K];
  if (!noise) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      dlogs[k] = clipd(z[k], -ION_LOG_CAP, ION_LOG_CAP);
      out.size = nanmax(out.size, fabs(dlogs[k]));
    }
  }
  double xn[3] = {0.0, 0.0, 0.0};
  const double capV = CAP_V * Vt;
  const bool want_J = !noise;
  const double QL = Q * L.L;
  // right-to-left current accumulators (see `Current` above), per carrier s (0 n, 1 p)
  double single[2] = {0.0, 0.0}, cqT[2] = {0.0, 0.0}, Tsum[2] = {0.0, 0.0};
  double bH[2] = {0.0, 0.0}, corr[2] = {0.0, 0.0};
  double Hs = 0.0, dtot = 0.0;
  // what the last iteration left for point i+1 (initially the right contact, point NP+1)
  Pt pr;
  contact(L, 1, Vint, pr);
  pr.n = exp(pr.lnn); pr.p = exp(pr.lnp);
  pr.offn = L.st(NP + 1, S_OFFN); pr.offp = L.st(NP + 1, S_OFFP);
  double R_r = 0.0;                 // bulk recombination of point i+1
  double Ri_r[2] = {0.0, 0.0};      // interface recombination of point i+1 (partial, then final)
  double q_r[2] = {0.0, 0.0};       // exp(sn Vg / V_T) / mu of point i+1
  double h_r = 0.0, dx_r = 0.0;     // interval i+1's h and dx
  int ifk_r = -2;                   // interval i+1's S_IFK
  double U_rr[2] = {0.0, 0.0};      // U of point i+2 (final)
  double Ri_rr[2] = {0.0, 0.0};     // interface recombination of point i+2 (final)

  for (int i = NP; i >= 0; --i) {
    Pt pi;
    if (i >= 1) {
      double x[3];
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        double v = *L.cd(i, 9 + r);
        if (!noise) {
#pragma unroll
          for (int k = 0; k < K; ++k) v -= *L.cd(i, 12 + r * K + k) * z[k];
        }
        x[r] = v - (*L.cd(i, r * 3 + 0) * xn[0] + *L.cd(i, r * 3 + 1) * xn[1] +
                    *L.cd(i, r * 3 + 2) * xn[2]);
      }
      xn[0] = x[0]; xn[1] = x[1]; xn[2] = x[2];
      const double yV = *L.y(0, i, 0), yN = *L.y(0, i, 1), yP = *L.y(0, i, 2);
      if (noise) {
        const double en = exp(yN), ep = exp(yP);
        out.size = nanmax(out.size, fabs(x[0]) * iVt);
        out.size = nanmax(out.size, fabs(x[1]) * (en / (en + L.nfloor)));
        out.size = nanmax(out.size, fabs(x[2]) * (ep / (ep + L.nfloor)));
        continue;
      }
      // damping: the caps, and densities below n_floor stepped in n (`density_steps`)
      const double sV = clipd(x[0], -capV, capV);
      double sd[2];
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const double yy = s == 0 ? yN : yP;
        const double d = x[1 + s];
        const bool below = yy < L.lognf;
        const bool pos = d > -1.0;
        double in_n = pos ? log1p(below ? d : 0.0) : -CAP_LN;
        in_n = clipd(in_n, -FLOOR_DROP_CAP, CAP_LN);
        sd[s] = below ? in_n : clipd(d, -CAP_LN, CAP_LN);
      }
      pi.V = yV + sV; pi.lnn = yN + sd[0]; pi.lnp = yP + sd[1];
      *L.y(0, i, 0) = pi.V; *L.y(0, i, 1) = pi.lnn; *L.y(0, i, 2) = pi.lnp;
      pi.n = exp(pi.lnn); pi.p = exp(pi.lnp);
      out.size = nanmax(out.size, fabs(sV) * iVt);
      out.size = nanmax(out.size, fabs(sd[0]) * (pi.n / (pi.n + L.nfloor)));
      out.size = nanmax(out.size, fabs(sd[1]) * (pi.p / (pi.p + L.nfloor)));
      out.finite = out.finite && isfinite(pi.V) && isfinite(pi.lnn) && isfinite(pi.lnp);
    } else {
      if (noise) break;
      contact(L, 0, Vint, pi);
      pi.n = exp(pi.lnn); pi.p = exp(pi.lnp);
    }
    pi.offn = L.st(i, S_OFFN); pi.offp = L.st(i, S_OFFP);
    // interval i (points i, i+1, both new): its traps' recombination at either end
    const double h_i = L.st(i, S_H), dx_i = L.st(i, S_DX);
    const int ifk_i = (int)L.st(i, S_IFK);
    double Ri_i[2] = {0.0, 0.0};
    if (ifk_i >= 0) {
      Iface t;
      iface_edge(L, ifk_i, pi.n, pr.n, pi.p, pr.p, t, false);
      Ri_i[0] = t.v[0]; Ri_i[1] = t.v[2];
      Ri_r[0] += t.v[1]; Ri_r[1] += t.v[3];
    }
    // the differential form: interval i's flux; an interface takes the interval before it
    double Jd[2] = {0.0, 0.0};
    if (L.currdiff) {
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const double sn = s == 0 ? -1.0 : 1.0;
        const double Vga = pi.V + (s == 0 ? pi.offn : pi.offp);
        const double Vgb = pr.V + (s == 0 ? pr.offn : pr.offp);
        double Bf, Bb, d1, d2;
        bern_pair(sn * (Vgb - Vga) * iVt, L.simss, Bf, Bb, d1, d2);
        const double da = s == 0 ? pi.n : pi.p, db = s == 0 ? pr.n : pr.p;
        const double mu = L.st(i, s == 0 ? S_MUN : S_MUP);
        Jd[s] = sn * Q * mu * Vt * (db * Bb - da * Bf) / (L.L * h_i);
      }
      if (ifk_i < -1) dtot += h_i * (Jd[0] + Jd[1]);
    }
    // point i+1 is final: finalise it (left interval i, right interval i+1)
    if (i + 1 <= NP) {
      const double Ug = L.st(i + 1, S_G) * gfrac;
      const double ck = 0.5 * (dx_i + dx_r);
      Hs += h_r;
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const double sn = s == 0 ? -1.0 : 1.0;
        const double Uk = R_r + Ri_r[s] - Ug;
        Tsum[s] += 0.5 * dx_r * (Uk + U_rr[s]);
        single[s] += ck * q_r[s];
        cqT[s] += ck * q_r[s] * Tsum[s];
        const double bk = sn * QL * h_r * Uk;
        bH[s] += bk * Hs;
        if (ifk_r >= -1) {
          const double tk = sn * 0.5 * QL * h_r * (Ri_r[s] + Ri_rr[s]);
          corr[s] += h_r * (bk - tk);
          if (L.currdiff) dtot += h_r * (Jd[s] + tk);
        }
        U_rr[s] = Uk;
        Ri_rr[s] = Ri_r[s];
      }
    }
    // point i becomes "point i+1" of the next iteration
    if (i >= 1) {
      double R, d1, d2;
      recomb(L, i, pi.n, pi.p, R, d1, d2);
      R_r = R;
    } else {
      R_r = 0.0;
    }
    q_r[0] = exp(-(pi.V + pi.offn) * iVt) / L.st(i, S_MUN);
    q_r[1] = exp((pi.V + pi.offp) * iVt) / L.st(i, S_MUP);
    Ri_r[0] = Ri_i[0]; Ri_r[1] = Ri_i[1];
    h_r = h_i; dx_r = dx_i; ifk_r = ifk_i;
    pr = pi;
  }
  if (want_J) {
    // point 0, the left contact: U = 0, no width term
    const double ck = 0.5 * dx_r;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      Tsum[s] += 0.5 * dx_r * (0.0 + U_rr[s]);
      single[s] += ck * q_r[s];
      cqT[s] += ck * q_r[s] * Tsum[s];
    }
    const double H = L.Hsum;
    double tot = 0.0;
    if (!L.currdiff) {
      Pt c0, cN;
      contact(L, 0, Vint, c0);
      contact(L, 1, Vint, cN);
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const double sn = s == 0 ? -1.0 : 1.0;
        const double dbl = Tsum[s] * single[s] - cqT[s];
        const double off0 = L.st(0, s == 0 ? S_OFFN : S_OFFP);
        const double offN = L.st(NP + 1, s == 0 ? S_OFFN : S_OFFP);
        const double d0 = exp(s == 0 ? c0.lnn : c0.lnp), dN = exp(s == 0 ? cN.lnn : cN.lnp);
        const double Kc = (Vt * (sn * dN * exp(sn * (cN.V + offN) * iVt) -
                                 sn * d0 * exp(sn * (c0.V + off0) * iVt)) -
                           sn * dbl) / single[s];
        tot += Q * Kc * H + bH[s] - corr[s];
      }
    } else {
      tot = dtot;
    }
    out.J = -L.left * tot / H;
  } else {
    out.J = 0.0;
  }
  if (!noise) {
#pragma unroll
    for (int k = 0; k < K; ++k) logs[k] += dlogs[k];
  }
  return out;
}

// ------------------------------------------------------------------------------------ start

// A point's potential and its mobile ions' densities only (the Poisson start and the ions'
// normalisations need no more of it).
__device__ __forceinline__ void pt_ions(const Lane& L, Pt& P, int k, const double* logs) {
  P.sl = slots_at(L, k);
  P.da = P.sl.a >= 0 ? exp(logs[P.sl.a] + P.V * L.iVt) : 0.0;
  P.dc = P.sl.c >= 0 ? exp(logs[L.ka + P.sl.c] - P.V * L.iVt) : 0.0;
}

// The normalisations that put each slot's ions into its region at the potential of the
// iterate (`_ion_logs`, solver.py:1695-1725, Boltzmann ions: closed form).
template <int K>
__device__ void ion_logs(const Lane& L, double Vint, double* logs) {
  double zero[K], num[K];
#pragma unroll
  for (int k = 0; k < K; ++k) { zero[k] = 0.0; num[k] = 0.0; }
  Pt a, b;
  contact(L, 0, Vint, a);
  pt_ions(L, a, 0, zero);
  for (int e = 0; e <= L.NP; ++e) {
    if (e + 1 <= L.NP) b.V = *L.y(0, e + 1, 0);
    else contact(L, 1, Vint, b);
    pt_ions(L, b, e + 1, zero);
    ion_edge<K>(L, a, b, L.st(e, S_H) * L.L, num);
    a = b;
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const double tk = L.total(k);
    logs[k] = tk > 0.0 ? log(tk / num[k]) : 0.0;
  }
}

// One Newton step of Poisson's equation alone, the densities following the potential and the
// ions re-fitted to it (`_poisson_delta`, solver.py:1757-1800; `_poisson_solve`,
// batch.py:486-503): a scalar tridiagonal system bordered by the slots, solved with the same
// forward-carried border as the Newton step. Without mobile ions each point's step is clipped
// to 10 V_T; with them the step is scaled as a whole (its largest entry m to V_T ln(1 + m/V_T)).
// Returns max |dV| / V_T of the step taken.
template <int K>
__device__ double poisson_step(Lane& L, double Vint, bool coupled, double* logs) {
  const int NP = L.NP;
  const double iVt = L.iVt;
  ion_logs<K>(L, Vint, logs);
  bool mobile = false;
#pragma unroll
  for (int k = 0; k < K; ++k) mobile = mobile || L.total(k) > 0.0;
  mobile = mobile && coupled;
  Pt pm, pc, pn;
  contact(L, 0, Vint, pm);
  pt_ions(L, pm, 0, logs);
  pc.V = *L.y(0, 1, 0); pc.lnn = *L.y(0, 1, 1); pc.lnp = *L.y(0, 1, 2);
  pt_ions(L, pc, 1, logs);
  double num[K], wp[K], dU[K], Sm[K][K], sv[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    num[k] = 0.0; wp[k] = 0.0; dU[k] = 0.0; sv[k] = 0.0;
#pragma unroll
    for (int j = 0; j < K; ++j) Sm[k][j] = 0.0;
  }
  double h_m = L.st(0, S_H);
  ion_edge<K>(L, pm, pc, h_m * L.L, num);
  double cprev = 0.0, dF = 0.0;
  for (int i = 1; i <= NP; ++i) {
    if (i < NP) { pn.V = *L.y(0, i + 1, 0); pn.lnn = *L.y(0, i + 1, 1); pn.lnp = *L.y(0, i + 1, 2); }
    else contact(L, 1, Vint, pn);
    pt_ions(L, pn, i + 1, logs);
    const double h_i = L.st(i, S_H);
    ion_edge<K>(L, pc, pn, h_i * L.L, num);
    const double facl = L.st(i, S_FACL), facm = L.st(i, S_FACM), facu = L.st(i, S_FACU);
    const double sP = L.st(i, S_SP);
    const double n = exp(pc.lnn), p = exp(pc.lnp);
    const double F = (facl * pm.V + facm * pc.V + facu * pn.V -
                      Q * (n - p + L.st(i, S_DOP) + L.afix(i) + pc.da - L.cfix(i) - pc.dc)) * sP;
    const double mid = (facm - Q * (n + p) * iVt - Q * (pc.da + pc.dc) * iVt) * sP;
    const double lo = i > 1 ? facl * sP : 0.0;
    const double up = i < NP ? facu * sP : 0.0;
    double U[K], W[K];
#pragma unroll
    for (int k = 0; k < K; ++k) U[k] = 0.0;
    if (pc.sl.a >= 0) U[pc.sl.a] = -Q * pc.da * sP;
    if (pc.sl.c >= 0) U[L.ka + pc.sl.c] = Q * pc.dc * sP;
    ion_w<K>(L, pm, pc, pn, h_m * L.L, h_i * L.L, W);
    const double im = 1.0 / (mid - lo * cprev);
#pragma unroll
    for (int k = 0; k < K; ++k) wp[k] = W[k] - cprev * wp[k];
    dF = (-F - lo * dF) * im;
#pragma unroll
    for (int k = 0; k < K; ++k) dU[k] = (U[k] - lo * dU[k]) * im;
    cprev = up * im;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      sv[k] += wp[k] * dF;
#pragma unroll
      for (int j = 0; j < K; ++j) Sm[k][j] += wp[k] * dU[j];
    }
    *L.cd(i, 0) = cprev;
    *L.cd(i, 1) = dF;
#pragma unroll
    for (int k = 0; k < K; ++k) *L.cd(i, 2 + k) = dU[k];
    pm = pc; pc = pn; h_m = h_i;
  }
  double z[K];
#pragma unroll
  for (int k = 0; k < K; ++k) z[k] = 0.0;
  if (mobile) {
    double Msch[K][K], rr[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const double tk = L.total(k);
      const bool has = tk > 0.0;
      const double g = has ? num[k] / tk - 1.0 : 0.0;
      const double Dk = has ? num[k] / tk : 1.0;
#pragma unroll
      for (int j = 0; j < K; ++j) Msch[k][j] = (j == k ? Dk : 0.0) - Sm[k][j];
      rr[k] = -g - sv[k];
    }
    small_solve<K>(Msch, rr, z);
  }
  const double capV = CAP_V * L.Vt;
  double x = 0.0, m = 0.0, size = 0.0;
  for (int i = NP; i >= 1; --i) {
    double v = *L.cd(i, 1);
#pragma unroll
    for (int k = 0; k < K; ++k) v -= *L.cd(i, 2 + k) * z[k];
    x = v - *L.cd(i, 0) * x;
    if (mobile) {
      *L.cd(i, 1) = x;
      m = nanmax(m, fabs(x) * iVt);
    } else {
      const double dV = clipd(x, -capV, capV);
      *L.y(0, i, 0) += dV;
      *L.y(0, i, 1) += dV * iVt;
      *L.y(0, i, 2) -= dV * iVt;
      size = nanmax(size, fabs(dV * iVt));
    }
  }
  if (mobile) {
    const double f = m > 0.0 ? fmin(log1p(m), CAP_V) / m : 1.0;
    for (int i = 1; i <= NP; ++i) {
      const double dV = *L.cd(i, 1) * f;
      *L.y(0, i, 0) += dV;
      *L.y(0, i, 1) += dV * iVt;
      *L.y(0, i, 2) -= dV * iVt;
      size = nanmax(size, fabs(dV * iVt));
    }
  }
  return size;
}

// The mobile ions of the iterate as fixed densities, no longer solved for (`_freeze`,
// batch.py:859-872).
template <int K>
__device__ void freeze(Lane& L, const double* logs) {
  for (int i = 1; i <= L.NP; ++i) {
    Pt P;
    P.V = *L.y(0, i, 0);
    pt_ions(L, P, i, logs);
    L.FX[((size_t)i * 2) * L.Bp + L.l] = L.afix(i) + P.da;
    L.FX[((size_t)i * 2 + 1) * L.Bp + L.l] = L.cfix(i) + P.dc;
  }
  L.frozen = true;
}

__device__ void copy_state(const Lane& L, int dst, int src) {
  for (int i = 1; i <= L.NP; ++i)
#pragma unroll
    for (int c = 0; c < 3; ++c) *L.y(dst, i, c) = *L.y(src, i, c);
}

template <int K>
__device__ __forceinline__ void copyv(double* d, const double* s) {
#pragma unroll
  for (int k = 0; k < K; ++k) d[k] = s[k];
}

template <int K>
__device__ __forceinline__ bool finitev(const double* s) {
  bool ok = true;
#pragma unroll
  for (int k = 0; k < K; ++k) ok = ok && isfinite(s[k]);
  return ok;
}

// ------------------------------------------------------------------------------------ kernel

struct Args {
  int B, Bp, npmax, ka, kc;
  const double* S;
  const double* C;
  const double* IFt;
  const double* Y0;
  const double* V;
  const int* voff;
  const int* vcnt;
  double* J;
  uint8_t* ok;
  int* its;
  int* status;
  int* steps;  // [3][Bp] or null
  double* Y;
  double* FX;
  double* CD;
  int ncd;
  double tol;
  int max_iter, start_iter, strict, simss, mode;
  // dd_newton_step
  double* logs_io;
  const double* vint;
  double share;
  double* size_out;
  double* J_out;
};

template <int K>
__device__ void lane_init(Lane& L, const Args& a, int l) {
  L.S = a.S; L.C = a.C; L.IFt = a.IFt; L.Bp = a.Bp; L.l = l;
  L.ka = a.ka; L.K = K;
  L.Vt = L.sc(C_VT); L.iVt = 1.0 / L.Vt; L.L = L.sc(C_L);
  L.V0 = L.sc(C_V0); L.VL = L.sc(C_VL); L.left = L.sc(C_LEFT);
  L.lnnL = L.sc(C_LNNL); L.lnpL = L.sc(C_LNPL); L.lnnR = L.sc(C_LNNR); L.lnpR = L.sc(C_LNPR);
  L.Jscale = L.sc(C_JSCALE); L.Gshunt = L.sc(C_GSHUNT); L.gfrac = L.sc(C_GFRAC);
  L.nfloor = L.sc(C_NFLOOR); L.lognf = log(L.nfloor); L.Hsum = L.sc(C_HSUM);
  L.NP = (int)L.sc(C_NP);
  L.currdiff = L.sc(C_CURRDIFF) > 0.0; L.simss = a.simss;
#pragma unroll
  for (int k = 0; k < K; ++k) L.tot[k] = L.sc(C_TOT0 + k);
  L.Y = a.Y; L.FX = a.FX; L.CD = a.CD; L.ncd = a.ncd;
  L.ybuf = (size_t)(a.npmax + 2) * 3 * a.Bp;
  L.frozen = false;
  L.share = 1.0;
}

enum Phase { PH_POISSON = 0, PH_NEWTON, PH_DONE };
enum Ctx {
  X_START_F = 0, X_STAGE, X_PRE, X_SCAN,          // solve_batch (batch.py:875-1006)
  X_JV_START, X_JV_STAGE, X_JV_PRE, X_JV_SCAN     // solve_jv (solver.py:2105-2245)
};

template <int K>
__global__ void __launch_bounds__(32) solve_kernel(Args a) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= a.B) return;
  Lane L;
  lane_init<K>(L, a, l);
  const bool jv = a.mode == DD_MODE_JV;
  const int voff = a.voff[l], nv = a.vcnt[l];
  const double* Vl = a.V + voff;
  const double pre_cond = L.sc(C_PRECOND) > 0.0, fix_ions = L.sc(C_FIXIONS) > 0.0;
  const double first = pre_cond ? L.sc(C_VPRE) : Vl[0];
  // the start: the initial guess into the iterate
  for (int i = 1; i <= L.NP; ++i)
#pragma unroll
    for (int c = 0; c < 3; ++c) *L.y(0, i, c) = __ldg(a.Y0 + ((size_t)i * 3 + c) * a.Bp + l);
  bool mobile = false;
#pragma unroll
  for (int k = 0; k < K; ++k) mobile = mobile || L.tot[k] > 0.0;

  double logs[K], lgA[K], lgB[K], lgC[K];
#pragma unroll
  for (int k = 0; k < K; ++k) { logs[k] = 0.0; lgA[k] = 0.0; lgB[k] = 0.0; lgC[k] = 0.0; }
  int phase = PH_POISSON, pit = 0;
  const int pcap = jv ? a.max_iter : a.start_iter;
  // the Newton solve in progress
  int ctx = 0, it = 0, cap = 0, adv = ADV_NONE;
  double Vint = first, ratio = 0.0;
  double hs[4], hJ[4];
  int nsz = 0;
  bool floor_known = false, pending_noise = false;
  double noise_floor = 0.0;
  // the program's flags
  bool ok_f = false, kept_f = false, solved = false, pre_ok = true, ok_c = false;
  int stage = 0;
  double before = 1.0;
  int k = 0, below = 0, last_keep = 0;
  double Vlast = first, Vbefore = first;
  int jcur = 0;
  if (!jv) {
    while (below < nv && Vl[below] < first) ++below;  // searchsorted, left
  }
  a.status[l] = DD_LANE_OK;

  auto begin = [&](int c, double v, double share, int cp_, int ad, double ra) {
    ctx = c; Vint = v; L.share = share; cap = cp_; adv = ad; ratio = ra;
    it = 0; nsz = 0; floor_known = false; pending_noise = false;
#pragma unroll
    for (int q = 0; q < 4; ++q) { hs[q] = INFINITY; hJ[q] = INFINITY; }
    phase = PH_NEWTON;
  };
  // the scan's next voltage (batch: outward from the pre-bias; jv: the caller's order)
  auto scan_begin = [&]() {
    if (k >= nv) { phase = PH_DONE; return; }
    if (!jv) {
      jcur = k < nv - below ? below + k : nv - 1 - k;
      const double v = Vl[jcur];
      if (k == 0 || k == nv - below) {
        Vlast = first; Vbefore = first;
        copyv<K>(logs, lgC); copyv<K>(lgA, lgC); copyv<K>(lgB, lgC);
        begin(X_SCAN, v, 1.0, a.max_iter, ADV_TURN, 0.0);
      } else {
        const double ra = Vlast != Vbefore ? (v - Vlast) / (Vlast - Vbefore) : 0.0;
#pragma unroll
        for (int q = 0; q < K; ++q)
          logs[q] = lgA[q] + (ra != 0.0 ? clipd(ra * (lgA[q] - lgB[q]), -ION_LOG_CAP, ION_LOG_CAP) : 0.0);
        begin(X_SCAN, v, 1.0, a.max_iter, last_keep ? ADV_KEEP : ADV_NOKEEP, ra);
      }
    } else {
      jcur = k;
      copyv<K>(logs, lgA);
      begin(X_JV_SCAN, Vl[k], 1.0, a.max_iter, last_keep ? ADV_KEEP : ADV_NOKEEP, 0.0);
    }
  };
  auto freeze_and_scan = [&]() {
    L.share = 1.0;
    if (!jv) {
      const bool fr = pre_cond && fix_ions;
      if (fr) freeze<K>(L, logs);
      pre_ok = pre_ok || !fr;
      copy_state(L, 3, 0);
      copyv<K>(lgC, logs);
      k = 0;
      scan_begin();
    } else {
      if (pre_cond && fix_ions) freeze<K>(L, logs);
      copyv<K>(lgA, logs);
      k = 0; last_keep = 1;  // the start is the carry
      scan_begin();
    }
  };
  auto batch_pre = [&]() {
    L.share = 1.0;
    if (solved) { pre_ok = true; freeze_and_scan(); }
    else begin(X_PRE, first, 1.0, a.start_iter, ADV_NONE, 0.0);
  };
  auto stage_begin = [&]() {
    const double share = c_stage_share[stage];
    const double sh = log(share / before);
#pragma unroll
    for (int q = 0; q < K; ++q) logs[q] += sh;
    if (!jv) { copy_state(L, 3, 0); copyv<K>(lgC, logs); }
    begin(jv ? X_JV_STAGE : X_STAGE, first, share, jv ? a.max_iter : a.start_iter, ADV_NONE, 0.0);
  };
  auto jv_pre = [&]() {
    L.share = 1.0;
    if (pre_cond) begin(X_JV_PRE, L.sc(C_VPRE), 1.0, a.max_iter, ADV_NONE, 0.0);
    else freeze_and_scan();
  };

  int n_border = 0, n_plain = 0;
  while (phase != PH_DONE) {
    if (phase == PH_POISSON) {
      const double size = poisson_step<K>(L, first, jv ? mobile : true, logs);
      ++pit;
      const bool stop = jv ? (size < POISSON_TOL || pit >= pcap) : (!(size > POISSON_TOL) || pit >= pcap);
      if (!stop) continue;
      ion_logs<K>(L, first, logs);
      if (!jv) {
        copy_state(L, 1, 0);
        copyv<K>(lgA, logs);
        begin(X_START_F, first, 1.0, a.start_iter, ADV_NONE, 0.0);
      } else if (mobile) {
        copy_state(L, 1, 0);
        copyv<K>(lgA, logs);
        begin(X_JV_START, first, 1.0, a.max_iter, ADV_NONE, 0.0);
      } else {
        jv_pre();
      }
      continue;
    }
    // ------------------------------------------------------------ one Newton step
    bool end = false, conv = false, fin = true;
    double Jv = 0.0;
    if (pending_noise) {
      const StepOut o = newton_step<K>(L, Vint, logs, ADV_NONE, 0.0, true);
      ++n_plain;
      noise_floor = o.size; floor_known = true; pending_noise = false;
      double mx = 0.0;
      for (int q = 4 - (nsz < 4 ? nsz : 4); q < 4; ++q) mx = nanmax(mx, hs[q]);
      if (mx < noise_floor) { end = true; conv = true; }
      else if (it >= cap) { end = true; conv = false; }
      Jv = hJ[3];
      fin = isfinite(Jv) || true;
      if (!end) continue;
    } else {
      const StepOut o = newton_step<K>(L, Vint, logs, adv, ratio, false);
      adv = ADV_NONE;
      ++it;
      bool border = false;
#pragma unroll
      for (int q = 0; q < K; ++q) border = border || L.total(q) > 0.0;
      if (border) ++n_border; else ++n_plain;
#pragma unroll
      for (int q = 0; q < 3; ++q) { hs[q] = hs[q + 1]; hJ[q] = hJ[q + 1]; }
      hs[3] = o.size; hJ[3] = o.J;
      ++nsz;
      Jv = o.J;
      fin = o.finite && finitev<K>(logs);
      const double size = o.size;
      const bool isn = size != size;
      const bool settle = ctx >= X_JV_START;
      if (!settle) {
        double mx = hs[0], mn = hs[1];
#pragma unroll
        for (int q = 1; q < 4; ++q) mx = nanmax(mx, hs[q]);
#pragma unroll
        for (int q = 2; q < 4; ++q) mn = (hs[q] < mn || hs[q] != hs[q]) ? hs[q] : mn;
        const bool stalled = it > STALL_STEPS && mx < ROUND_OFF_FLOOR && mn >= 0.1 * hs[0];
        double dJ = 0.0;
#pragma unroll
        for (int q = 0; q < 4; ++q) dJ = nanmax(dJ, fabs(hJ[q] - hJ[3]));
        const bool settled = it > STALL_STEPS && size < CURRENT_STEP_CAP &&
                             dJ < CURRENT_TOL * (L.Jscale + fabs(hJ[3]));
        const bool quad = it > 1 && size < QUADRATIC_TOL && size < QUADRATIC_RATIO * hs[2];
        conv = a.strict ? (size < a.tol || stalled) : (size < a.tol || stalled || settled || quad);
        end = conv || it >= cap || isn;
      } else {
        if (isn) { end = true; conv = false; }
        else {
          const int n4 = nsz < 4 ? nsz : 4;
          double mx = 0.0, mn = INFINITY;
          for (int q = 4 - n4; q < 4; ++q) mx = nanmax(mx, hs[q]);
          for (int q = 4 - n4 + 1; q < 4; ++q) mn = fmin(mn, hs[q]);
          bool done = size < a.tol || (nsz >= 4 && mx < ROUND_OFF_FLOOR && mn >= 0.1 * hs[0]);
          if (!done && nsz >= 4 && mx < NOISE_FLOOR_CAP) {
            if (!floor_known) { pending_noise = true; continue; }
            done = mx < noise_floor;
          }
          if (done) { end = true; conv = true; }
          else if (it >= cap) { end = true; conv = false; }
        }
      }
      if (!end) continue;
    }
    // ------------------------------------------------------------ a solve ended
    switch (ctx) {
      case X_START_F: {
        ok_f = conv; kept_f = fin;
        if (ok_f || !mobile) {
          if (!kept_f) { copy_state(L, 0, 1); copyv<K>(logs, lgA); }
          solved = ok_f;
          batch_pre();
        } else {
          copy_state(L, 2, 0); copyv<K>(lgB, logs);
          copy_state(L, 0, 1); copyv<K>(logs, lgA);
          before = 1.0; stage = 0;
          stage_begin();
        }
        break;
      }
      case X_STAGE: {
        ok_c = conv;
        if (!fin) { copy_state(L, 0, 3); copyv<K>(logs, lgC); }
        before = c_stage_share[stage];
        ++stage;
        if (stage < 4) { stage_begin(); break; }
        const bool staged = ok_c;
        if (!staged) {
          if (kept_f) { copy_state(L, 0, 2); copyv<K>(logs, lgB); }
          else { copy_state(L, 0, 1); copyv<K>(logs, lgA); }
        }
        solved = staged;
        batch_pre();
        break;
      }
      case X_PRE: {
        pre_ok = conv;
        freeze_and_scan();
        break;
      }
      case X_SCAN: {
        const int pos = voff + jcur;
        a.J[pos] = Jv + L.Gshunt * Vint;
        a.ok[pos] = (conv && pre_ok) ? 1 : 0;
        a.its[pos] = it;
        const bool keep = conv && fin;
        if (keep) {
          copyv<K>(lgB, lgA); copyv<K>(lgA, logs);
          Vbefore = Vlast; Vlast = Vint; last_keep = 1;
        } else {
          last_keep = 0;
        }
        ++k;
        scan_begin();
        break;
      }
      case X_JV_START: {
        if (conv) { jv_pre(); break; }
        copy_state(L, 0, 1); copyv<K>(logs, lgA);
        before = 1.0; stage = 0;
        stage_begin();
        break;
      }
      case X_JV_STAGE: {
        before = c_stage_share[stage];
        if (!conv) { copy_state(L, 0, 1); copyv<K>(logs, lgA); jv_pre(); break; }
        ++stage;
        if (stage < 4) stage_begin();
        else jv_pre();
        break;
      }
      case X_JV_PRE: {
        if (!conv) {
          a.status[l] = DD_LANE_PREBIAS_FAILED;
          for (int q = 0; q < nv; ++q) { a.J[voff + q] = NAN; a.ok[voff + q] = 0; a.its[voff + q] = 0; }
          phase = PH_DONE;
          break;
        }
        freeze_and_scan();
        break;
      }
      case X_JV_SCAN: {
        const int pos = voff + jcur;
        a.J[pos] = Jv + L.Gshunt * Vint;
        a.ok[pos] = conv ? 1 : 0;
        a.its[pos] = it;
        const bool keep = conv && fin;
        if (keep) { copyv<K>(lgA, logs); last_keep = 1; }
        else last_keep = 0;
        ++k;
        scan_begin();
        break;
      }
    }
  }
  if (a.steps) {
    a.steps[l] = n_border;
    a.steps[a.Bp + l] = n_plain;
    a.steps[2 * a.Bp + l] = pit;
  }
}

// One Newton step per lane from a given state (dd_newton_step).
template <int K>
__global__ void __launch_bounds__(32) step_kernel(Args a) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= a.B) return;
  Lane L;
  lane_init<K>(L, a, l);
  L.share = a.share;
  double logs[K];
#pragma unroll
  for (int k = 0; k < K; ++k) logs[k] = a.logs_io[(size_t)k * a.Bp + l];
  const StepOut o = newton_step<K>(L, a.vint[l], logs, ADV_NONE, 0.0, false);
#pragma unroll
  for (int k = 0; k < K; ++k) a.logs_io[(size_t)k * a.Bp + l] = logs[k];
  a.size_out[l] = o.size;
  a.J_out[l] = o.J;
}

}  // namespace dd

// ======================================================================================== C ABI

namespace {

int slots_k(const dd_batch* b) { return b->k_anion + b->k_cation <= 2 ? 2 : 4; }

size_t ws_elems(const dd_batch* b, size_t* y_e, size_t* fx_e, size_t* cd_e, int* ncd) {
  const int K = slots_k(b);
  *ncd = 12 + 3 * K;
  const size_t nodes = (size_t)b->np_max + 2;
  *y_e = (size_t)dd::DD_NBUF * nodes * 3 * b->lane_stride;
  *fx_e = nodes * 2 * b->lane_stride;
  *cd_e = nodes * (size_t)(*ncd) * b->lane_stride;
  return *y_e + *fx_e + *cd_e;
}

int check_batch(const dd_batch* b) {
  if (!b || !b->stat || !b->scal || !b->iface || !b->y0) return DD_ERR_ARGS;
  if (b->n_lanes < 1 || b->lane_stride < b->n_lanes || b->lane_stride % 32 != 0) return DD_ERR_ARGS;
  if (b->np_max < 3 || b->k_anion < 1 || b->k_cation < 1 || b->k_anion + b->k_cation > dd::DD_MAXK)
    return DD_ERR_ARGS;
  return DD_OK;
}

dd::Args make_args(const dd_batch* b, void* ws) {
  dd::Args a{};
  a.B = b->n_lanes; a.Bp = b->lane_stride; a.npmax = b->np_max;
  a.ka = b->k_anion; a.kc = b->k_cation;
  a.S = b->stat; a.C = b->scal; a.IFt = b->iface; a.Y0 = b->y0;
  size_t ye, fe, ce;
  int ncd;
  ws_elems(b, &ye, &fe, &ce, &ncd);
  double* base = static_cast<double*>(ws);
  a.Y = base; a.FX = base + ye; a.CD = base + ye + fe; a.ncd = ncd;
  return a;
}

}  // namespace

extern "C" {

int dd_abi_version(void) { return (1 << 16) | 0; }

const char* dd_status_string(int status) {
  switch (status) {
    case DD_OK: return "ok";
    case DD_ERR_ARGS: return "invalid arguments";
    case DD_ERR_WORKSPACE: return "workspace too small";
    case DD_ERR_LAUNCH: return "kernel launch failed";
    case DD_ERR_DEVICE: return "no sm_100 device";
    default: return "unknown status";
  }
}

int dd_workspace_bytes(const dd_batch* batch, size_t* bytes) {
  if (check_batch(batch) != DD_OK || !bytes) return DD_ERR_ARGS;
  size_t ye, fe, ce;
  int ncd;
  *bytes = ws_elems(batch, &ye, &fe, &ce, &ncd) * sizeof(double);
  return DD_OK;
}

int dd_solve(const dd_batch* batch, const dd_voltages* volts, const dd_opts* opts, double* J,
             uint8_t* converged, int32_t* iterations, int32_t* lane_status, int32_t* lane_steps,
             void* workspace, size_t workspace_bytes, void* stream) {
  int st = check_batch(batch);
  if (st != DD_OK) return st;
  if (!volts || !volts->v || !volts->offset || !volts->count || !opts || !J || !converged ||
      !iterations || !lane_status || !workspace)
    return DD_ERR_ARGS;
  if (opts->max_iter < 1 || opts->start_iter < 1 || (opts->mode != DD_MODE_BATCH && opts->mode != DD_MODE_JV) ||
      (opts->bernoulli != DD_BERNOULLI_EXACT && opts->bernoulli != DD_BERNOULLI_SIMSS) ||
      opts->precision != DD_PRECISION_FP64)
    return DD_ERR_ARGS;
  size_t need;
  dd_workspace_bytes(batch, &need);
  if (workspace_bytes < need) return DD_ERR_WORKSPACE;
  dd::Args a = make_args(batch, workspace);
  a.V = volts->v; a.voff = volts->offset; a.vcnt = volts->count;
  a.J = J; a.ok = converged; a.its = iterations; a.status = lane_status; a.steps = lane_steps;
  a.tol = opts->tol; a.max_iter = opts->max_iter; a.start_iter = opts->start_iter;
  a.strict = opts->strict; a.simss = opts->bernoulli == DD_BERNOULLI_SIMSS; a.mode = opts->mode;
  const dim3 grid((batch->lane_stride + 31) / 32), block(32);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (slots_k(batch) == 2) dd::solve_kernel<2><<<grid, block, 0, s>>>(a);
  else dd::solve_kernel<4><<<grid, block, 0, s>>>(a);
  return cudaGetLastError() == cudaSuccess ? DD_OK : DD_ERR_LAUNCH;
}

int dd_newton_step(const dd_batch* batch, double* y, double* logs, const double* vint,
                   double share, const dd_opts* opts, double* size, double* J, void* workspace,
                   size_t workspace_bytes, void* stream) {
  int st = check_batch(batch);
  if (st != DD_OK) return st;
  if (!y || !logs || !vint || !opts || !size || !J || !workspace) return DD_ERR_ARGS;
  size_t need;
  dd_workspace_bytes(batch, &need);
  if (workspace_bytes < need) return DD_ERR_WORKSPACE;
  dd::Args a = make_args(batch, workspace);
  a.Y = y;  // the caller's state is the iterate buffer
  a.simss = opts->bernoulli == DD_BERNOULLI_SIMSS;
  a.logs_io = logs; a.vint = vint; a.share = share; a.size_out = size; a.J_out = J;
  const dim3 grid((batch->lane_stride + 31) / 32), block(32);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (slots_k(batch) == 2) dd::step_kernel<2><<<grid, block, 0, s>>>(a);
  else dd::step_kernel<4><<<grid, block, 0, s>>>(a);
  return cudaGetLastError() == cudaSuccess ? DD_OK : DD_ERR_LAUNCH;
}

}  // extern "C"
