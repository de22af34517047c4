// Device-side physics shared by the solve (dd_solve.cu) and its adjoint (dd_adjoint.cu): the
// reference's constants and stops, the Bernoulli function, one interval's Scharfetter-Gummel
// fluxes, recombination, interface traps, the ions' numbers, and the per-lane view of the packed
// batch (`Lane`). Everything is inline: each translation unit gets its own copy. The helpers that
// read a node's static record take any lane view with Lane's members (`st`, `afix`, `cfix`, ...):
// the solve's sweeps pass one that reads the record from shared memory.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "dd_layout.h"

// The transcendental functions of the hot loops, as the including file wants them: inline by
// default; a file may define these first to route every call site through one shared copy.
#ifndef DD_EXP
#define DD_EXP(x) exp(x)
#endif
#ifndef DD_EXPM1
#define DD_EXPM1(x) expm1(x)
#endif
#ifndef DD_LOG1P
#define DD_LOG1P(x) log1p(x)
#endif

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
  const double e = DD_EXPM1(a);
  const double r = 1.0 / e;  // one reciprocal for both quotients
  b = a * r;
  db = (1.0 - b) * r - b;  // 1/e - a(e+1)/e^2, finite where e overflows
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

// Element i of a small register array (0 where i is outside 0 .. N-1), and the update of one
// element, by predicated selects over the array: an index known only at run time into a
// register array would move the whole array to local memory.
template <int N>
__device__ __forceinline__ double pick(const double* a, int i) {
  double v = 0.0;
#pragma unroll
  for (int q = 0; q < N; ++q) v = q == i ? a[q] : v;
  return v;
}
template <int N>
__device__ __forceinline__ void add_at(double* a, int i, double v) {
#pragma unroll
  for (int q = 0; q < N; ++q)
    if (q == i) a[q] += v;
}
template <int N>
__device__ __forceinline__ void set_at(double* a, int i, double v) {
#pragma unroll
  for (int q = 0; q < N; ++q)
    if (q == i) a[q] = v;
}

// ------------------------------------------------------------------------------------ lane

struct Lane {
  // batch
  const double* __restrict__ S;
  const double* __restrict__ C;
  const double* __restrict__ IFt;
  int Bp, l, NP, ka, K;
  double Vt, iVt, L, gfrac, nfloor, lognf;
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
  // the pair of threads that share this device: half 0 eliminates rows 1..mid-1 downwards
  // and owns points 1..mid, half 1 eliminates rows NP..mid+1 upwards and owns mid+1..NP
  int half, mid;
  unsigned mask;  // the pair's two lanes in the warp
  int base;       // warp lane of half 0

  __device__ __forceinline__ double st(int k, int f) const {
    return __ldg(S + ((size_t)k * DD_NF + f) * Bp + l);
  }
  __device__ __forceinline__ double sc(int f) const { return __ldg(C + (size_t)f * Bp + l); }
  // Scalars read once or twice per Newton step are read from the record when needed rather
  // than held in registers through the sweeps.
  __device__ __forceinline__ double V0() const { return sc(C_V0); }
  __device__ __forceinline__ double VL() const { return sc(C_VL); }
  __device__ __forceinline__ double left() const { return sc(C_LEFT); }
  __device__ __forceinline__ double lnnL() const { return sc(C_LNNL); }
  __device__ __forceinline__ double lnpL() const { return sc(C_LNPL); }
  __device__ __forceinline__ double lnnR() const { return sc(C_LNNR); }
  __device__ __forceinline__ double lnpR() const { return sc(C_LNPR); }
  __device__ __forceinline__ double Jscale() const { return sc(C_JSCALE); }
  __device__ __forceinline__ double Gshunt() const { return sc(C_GSHUNT); }
  __device__ __forceinline__ double Hsum() const { return sc(C_HSUM); }
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
  __device__ __forceinline__ double total(int k) const {
    return frozen ? 0.0 : share * pick<DD_MAXK>(tot, k);
  }
};

// Slot of a point for each species, -1 where the species is not mobile there (or frozen).
struct Slots {
  int a, c;
};

template <class LT>
__device__ __forceinline__ Slots slots_at(const LT& L, int k) {
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

// pt_fill with the K normalisations in registers (read by selects, `pick`).
template <int K, class LT>
__device__ __forceinline__ void pt_fill_k(const LT& L, Pt& P, int k, const double* logs) {
  P.n = DD_EXP(P.lnn);
  P.p = DD_EXP(P.lnp);
  P.offn = L.st(k, S_OFFN);
  P.offp = L.st(k, S_OFFP);
  P.sl = slots_at(L, k);
  P.da = P.sl.a >= 0 ? DD_EXP(pick<K>(logs, P.sl.a) + P.V * L.iVt) : 0.0;
  P.dc = P.sl.c >= 0 ? DD_EXP(pick<K>(logs, L.ka + P.sl.c) - P.V * L.iVt) : 0.0;
}

// The contacts' states (`_bounds`, batch.py:255-259).
__device__ __forceinline__ void contact(const Lane& L, int right, double Vint, Pt& P) {
  if (!right) { P.V = L.V0() + 0.5 * L.left() * Vint; P.lnn = L.lnnL(); P.lnp = L.lnpL(); }
  else { P.V = L.VL() - 0.5 * L.left() * Vint; P.lnn = L.lnnR(); P.lnp = L.lnpR(); }
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
template <class LT>
__device__ __forceinline__ void recomb(const LT& L, int k, double n, double p, double& R,
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
    // one reciprocal for the three quotients (an FP64 division is a long instruction sequence)
    const double iden = 1.0 / den;
    const double srh = kk * (n * p - nt0 * pt0) * iden;
    R += srh;
    dRn += n * (kk * p - srh * Cn) * iden;
    dRp += p * (kk * n - srh * Cp) * iden;
  }
}

// Interface traps of one interval (table row t), steady state, one level (solver.py:814-850):
// v = (Rn_L, Rn_R, Rp_L, Rp_R, Q) and, when asked, their derivatives in ln nL, ln nR, ln pL, ln pR.
struct Iface {
  double v[5];
  double d[4][5];
};

static __device__ void iface_edge(const Lane& L, int t, double nL, double nR, double pL, double pR,
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
  if (a.sl.a >= 0 && a.sl.a == b.sl.a) add_at<K>(num, a.sl.a, 0.5 * (a.da + b.da) * hL);
  if (a.sl.c >= 0 && a.sl.c == b.sl.c) add_at<K>(num, L.ka + a.sl.c, 0.5 * (a.dc + b.dc) * hL);
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
      set_at<K>(W, k, wpt * pc.da * L.iVt / tk);
    }
  }
  if (pc.sl.c >= 0) {
    const int k = L.ka + pc.sl.c;
    const double tk = L.total(k);
    if (tk > 0.0) {
      const double wpt = 0.5 * ((pm.sl.c == pc.sl.c ? hLm : 0.0) + (pn.sl.c == pc.sl.c ? hLp : 0.0));
      set_at<K>(W, k, -wpt * pc.dc * L.iVt / tk);
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

// ------------------------------------------------------------------------------------ rows

// Row i's residual and blocks (`_assemble`, solver.py:1021-1187, the supported scope) from its
// points (i-1, i, i+1) and intervals (left el, right er): A, B, C in (V, ln n, ln p), the
// right-hand side -F (or, with `noise`, each row's round-off eps sum |dF/dy| |y|, `_noise_step`),
// the ion columns U (Poisson row only) and the constraints' border W (potential only).
//
// In the mirrored frame of half 1 (nodes taken from NP down, `mirror`) "behind" (pm) is the
// physical right neighbour and "ahead" (pn) the left one: the fluxes are evaluated in that order
// (which turns their sign, as the mirrored equations want), the Poisson stencil's two sides swap
// (fL, fU), and A couples to the point behind, C to the one ahead, as in the unmirrored frame.
// Only the interface traps, which know their physical left and right, read `mirror`.
template <int K, class LT>
__device__ __forceinline__ void assemble_row(const LT& L, int i, const Pt& pm, const Pt& pc,
                                             const Pt& pn, const Flux& el, const Flux& er,
                                             double hm, double hp, int ifk_m, int ifk_i,
                                             bool noise, bool mirror, double (&A)[3][3],
                                             double (&Bm)[3][3], double (&Cm)[3][3],
                                             double (&rhs)[3], double (&U0)[K], double (&W)[K]) {
  const double iVt = L.iVt;
  const double facl = L.st(i, mirror ? S_FACU : S_FACL), facm = L.st(i, S_FACM);
  const double facu = L.st(i, mirror ? S_FACL : S_FACU);
  const double fac = L.st(i, S_FAC), sP = L.st(i, S_SP), sC = L.st(i, S_SC);
  double R, dRn, dRp;
  recomb(L, i, pc.n, pc.p, R, dRn, dRp);
  const double gen = L.st(i, S_G) * L.gfrac;
  double elec = hm * er.Fn - hp * el.Fn + fac * (gen - R);
  double hole = hp * el.Fp - hm * er.Fp + fac * (gen - R);
  double pois = facl * pm.V + facm * pc.V + facu * pn.V -
                Q * (pc.n - pc.p + L.st(i, S_DOP) + L.afix(i) + pc.da - L.cfix(i) - pc.dc);
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
    const double sc3[3] = {Q * sP, -fac * sC, -fac * sC};
    double X[3] = {0.0, 0.0, 0.0};
    Iface t;
    // (value, derivative in this point's own ln n / ln p, in the other end's) of an interval
    // whose physical left end is `left_is_me ? pc : other`
    auto add = [&](int ifk, const Pt& other, bool left_is_me, double (&Oth)[3][3]) {
      if (left_is_me) iface_edge(L, ifk, pc.n, other.n, pc.p, other.p, t, true);
      else iface_edge(L, ifk, other.n, pc.n, other.p, pc.p, t, true);
      const int lo[3] = {4, 0, 2}, hi[3] = {4, 1, 3};
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const int q = left_is_me ? lo[r] : hi[r];
        const int dn_me = left_is_me ? 0 : 1, dp_me = left_is_me ? 2 : 3;
        X[r] += t.v[q];
        Bm[r][1] += sc3[r] * t.d[dn_me][q];
        Bm[r][2] += sc3[r] * t.d[dp_me][q];
        Oth[r][1] += sc3[r] * t.d[1 - dn_me][q];
        Oth[r][2] += sc3[r] * t.d[5 - dp_me][q];
      }
    };
    if (ifk_m >= 0) add(ifk_m, pm, mirror, A);    // the interval behind this point
    if (ifk_i >= 0) add(ifk_i, pn, !mirror, Cm);  // the interval ahead of it
    pois += Q * X[0];
    elec -= fac * X[1];
    hole -= fac * X[2];
  }
  if (!noise) {
    rhs[0] = -pois * sP; rhs[1] = -elec * sC; rhs[2] = -hole * sC;
#pragma unroll
    for (int k = 0; k < K; ++k) U0[k] = 0.0;
    if (pc.sl.a >= 0) set_at<K>(U0, pc.sl.a, -Q * pc.da * sP);
    if (pc.sl.c >= 0) set_at<K>(U0, L.ka + pc.sl.c, Q * pc.dc * sP);
    ion_w<K>(L, pm, pc, pn, hm * L.L, hp * L.L, W);
  } else {
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
}

// The inverse of a 3x3 block by its adjugate (jaxdd's choice, `_inverse3`, solver.py:1481-1495).
__device__ __forceinline__ void inv3(const double (&M)[3][3], double (&Mi)[3][3]) {
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
  Mi[0][0] = co00 * idet; Mi[0][1] = co01 * idet; Mi[0][2] = co02 * idet;
  Mi[1][0] = co10 * idet; Mi[1][1] = co11 * idet; Mi[1][2] = co12 * idet;
  Mi[2][0] = co20 * idet; Mi[2][1] = co21 * idet; Mi[2][2] = co22 * idet;
}

}  // namespace dd
