// The small-signal admittance of a batch about its steady states on sm_100a: jaxdd's
// `solve_impedance` for devices without mobile ions (src/jaxdd/impedance.py:230-409).
//
// At a steady state y0 a small voltage dV e^{iwt} drives (J + iw M) dy = -dF/dV dV: J the steady
// Jacobian (the solve's own blocks), M the time terms of implicit Euler (-fac n sC and -fac p sC
// on each continuity row's own ln n, ln p), and the traps' occupations as states with their own
// rates (`_trap_blocks`, `_interface_blocks`: the occupation beyond its instantaneous response,
// -iw/(iw + a) of it, in the rates and the charge). One complex block-tridiagonal solve per
// (device, frequency), then the current of a time step (SIMsalabim's integral form over each
// point's control volume, each density's change and the displacement current, `_current_parts`
// with `tr`, batch.py:316-403) linearised in dy, the voltage and the traps' extra rates:
// Y = dJ/dV = J'(0) + iw (J'(1) - J'(0)) + J_u (`_admittance`'s `current`, impedance.py:338-350).
//
// How: a first kernel takes one device and keeps, per node, the steady blocks A, B, C, the mass
// terms, the bulk traps' rate, drive and capture terms, and the current's steady integrands; a
// second takes one (device, frequency) pair per thread (a grid-stride loop over all pairs): the
// complex elimination forward, the back substitution, then one left-to-right pass that carries
// the current's tangent (its dt-free and its per-dt parts at once) to the admittance. jaxdd
// differentiates its current with jax.jvp; the tangent here is written out.
#include <cuda_runtime.h>
#include <stdint.h>

#include "dd_launch.h"
#include "dd_layout.h"
#include "dd_physics.cuh"
#include "dd_time.cuh"
#include "../../include/jaxdd_b200.h"

namespace dd {
namespace imp {

struct cplx {
  double re, im;
};
__device__ __forceinline__ cplx mk(double r, double i = 0.0) { return cplx{r, i}; }
__device__ __forceinline__ cplx operator+(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cplx operator-(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ cplx operator*(cplx a, cplx b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ cplx operator*(double s, cplx a) { return {s * a.re, s * a.im}; }
__device__ __forceinline__ cplx operator/(cplx a, cplx b) {
  // Smith's division
  if (fabs(b.re) >= fabs(b.im)) {
    const double r = b.im / b.re, den = b.re + b.im * r;
    return {(a.re + a.im * r) / den, (a.im - a.re * r) / den};
  }
  const double r = b.re / b.im, den = b.re * r + b.im;
  return {(a.re * r + a.im) / den, (a.im * r - a.re) / den};
}

// (df - df0)/df0 of a trap level of rate `a` at `lap` (jaxdd `_step_transfer`,
// impedance.py:107-117), in its rates (hr) and its charge (hc): continuous both -lap/(lap + a);
// over implicit Euler's steps of dt (lap then (1 - 1/z)/dt) the occupation's mean over a step
// and its value at the step's end.
__device__ __forceinline__ void transfer(double a, cplx lap, double dt, cplx& hr, cplx& hc) {
  if (!(dt > 0.0)) {
    hr = mk(0.0) - lap / (lap + mk(a));
    hc = hr;
    return;
  }
  const double x = a * dt, E = exp(-x), m = -expm1(-x) / x;
  const cplx den = mk(1.0) - E * (mk(1.0) - dt * lap);
  hr = ((-m * dt) * lap) / den;
  hc = ((-E * dt) * lap) / den;
}

// Per node of the steady-state record (first kernel's output), [node][word][lane].
enum {
  P_A = 0, P_B = 9, P_C = 18,      // the steady blocks
  P_MN = 27, P_MP,                 // the mass terms -fac n sC, -fac p sC
  P_TA, P_TDN, P_TDP, P_TRN, P_TRP, // bulk traps: rate a, drive in ln n / ln p, dR_n, dR_p
  P_EVN, P_EVP, P_IUN, P_IUP,      // exp(-+Vg/V_T), the integrated recombination
  P_DRN, P_DRP,                    // n dR/dn, p dR/dp
  P_N, P_P,                        // the densities
  P_WORDS
};
// Per lane scalars: single_n, single_p, K_n, K_p.
enum { L_SN = 0, L_SP, L_KN, L_KP, L_WORDS };
// Per node of a (device, frequency) thread: c' (9 complex) and d' (3 complex; then dy).
enum { W_C = 0, W_D = 18, W_WORDS = 24 };

struct Args {
  int B, Bp, npmax, ka, simss, nf;
  int K;  // ion slots, anion slots first (2 .. DD_MAXK; the ions' kernels)
  double dt;  // > 0: implicit Euler's steps of dt (the traps' step response); 0: continuous
  const double* S;
  const double* C;
  const double* IFt;
  const double* state;   // [np+2][3][Bp]
  const double* eps;     // [np+2][Bp]
  const double* vint;    // [Bp]
  const double* laps;    // [nf][2]: i omega
  double* rec;           // [np+2][P_WORDS][Bp]
  double* lsc;           // [L_WORDS][Bp]
  double* scr;           // [np+2][W_WORDS][T]
  double* Y;             // [nf][2][Bp]
  long T;
};

__device__ void lane_init(Lane& L, const Args& a, int l) {
  L.S = a.S; L.C = a.C; L.IFt = a.IFt; L.Bp = a.Bp; L.l = l; L.ka = a.ka; L.K = 2;
  L.Vt = L.sc(C_VT); L.iVt = 1.0 / L.Vt; L.L = L.sc(C_L);
      L.gfrac = L.sc(C_GFRAC);
  L.nfloor = L.sc(C_NFLOOR); L.lognf = log(L.nfloor);   L.NP = (int)L.sc(C_NP);
  L.mid = 0; L.currdiff = 0; L.simss = a.simss;
  L.tot[0] = 0.0; L.tot[1] = 0.0;
  L.FX = nullptr; L.CD = nullptr; L.ncd = 0; L.ybuf = 0;
  L.frozen = false;  // the devices have no mobile ions (the host refuses others): fixed ions
  L.share = 1.0;     // and slots come from the record
  L.half = 0; L.base = 0; L.mask = 0;
  L.Y = const_cast<double*>(a.state);
}

__device__ __forceinline__ void point(const Lane& L, int k, double Vint, Pt& P) {
  const double zero[2] = {0.0, 0.0};
  if (k == 0) contact(L, 0, Vint, P);
  else if (k == L.NP + 1) contact(L, 1, Vint, P);
  else { P.V = *L.y(0, k, 0); P.lnn = *L.y(0, k, 1); P.lnp = *L.y(0, k, 2); }
  pt_fill(L, P, k, zero);
}

// The steady state's blocks, mass and trap terms and the current's integrands, per node.
__global__ void __launch_bounds__(64) prepare_kernel(Args a) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= a.B) return;
  Lane L;
  lane_init(L, a, l);
  const int NP = L.NP;
  const double Vint = a.vint[l];
  auto rec = [&](int k, int f) -> double& { return a.rec[((size_t)k * P_WORDS + f) * a.Bp + l]; };
  Pt pm, pc, pn;
  point(L, 0, Vint, pm);
  point(L, 1, Vint, pc);
  Flux el, er;
  flux(L, pm, pc, L.st(0, S_MUN), L.st(0, S_MUP), el);
  for (int i = 1; i <= NP; ++i) {
    point(L, i + 1, Vint, pn);
    flux(L, pc, pn, L.st(i, S_MUN), L.st(i, S_MUP), er);
    double A[3][3], Bm[3][3], Cm[3][3], rhs[3], U0[2], W[2];
    assemble_row<2>(L, i, pm, pc, pn, el, er, L.st(i - 1, S_H), L.st(i, S_H),
                    (int)L.st(i - 1, S_IFK), (int)L.st(i, S_IFK), false, false, A, Bm, Cm, rhs,
                    U0, W);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        rec(i, P_A + 3 * r + c) = A[r][c];
        rec(i, P_B + 3 * r + c) = Bm[r][c];
        rec(i, P_C + 3 * r + c) = Cm[r][c];
      }
    const double fac = L.st(i, S_FAC), sC = L.st(i, S_SC);
    rec(i, P_MN) = -fac * pc.n * sC;
    rec(i, P_MP) = -fac * pc.p * sC;
    // bulk traps (`_trap_terms`, one neutral level)
    const double Nt = L.st(i, S_NT);
    double ta = 1.0, tdn = 0.0, tdp = 0.0, trn = 0.0, trp = 0.0;
    if (Nt > 0.0) {
      const double Cn = L.st(i, S_CNT), Cp = L.st(i, S_CPT), nt0 = L.st(i, S_NT0), pt0 = L.st(i, S_PT0);
      ta = Cn * (pc.n + nt0) + Cp * (pc.p + pt0);
      const double f = (Cn * pc.n + Cp * pt0) / ta;
      tdn = Cn * pc.n * (1.0 - f);
      tdp = -f * Cp * pc.p;
      trn = -Nt * Cn * (pc.n + nt0);
      trp = Nt * Cp * (pc.p + pt0);
    }
    rec(i, P_TA) = ta; rec(i, P_TDN) = tdn; rec(i, P_TDP) = tdp; rec(i, P_TRN) = trn; rec(i, P_TRP) = trp;
    pm = pc; pc = pn; el = er;
  }
  // the current's integrands (steady values) on the points 0..NP+1
  double iu[2] = {0.0, 0.0}, uc_prev[2] = {0.0, 0.0}, dx_prev = 0.0;
  double sgl[2] = {0.0, 0.0}, dbl[2] = {0.0, 0.0};
  // interface point recombination of point k: edges k-1 (right end) and k (left end)
  auto ri_at = [&](int k, double& rn, double& rp) {
    rn = 0.0; rp = 0.0;
    for (int e = k - 1; e <= k; ++e) {
      if (e < 0 || e > NP) continue;
      const int t = (int)L.st(e, S_IFK);
      if (t < 0) continue;
      Pt p0, p1;
      point(L, e, Vint, p0);
      point(L, e + 1, Vint, p1);
      Iface f;
      iface_edge(L, t, p0.n, p1.n, p0.p, p1.p, f, false);
      if (e == k) { rn += f.v[0]; rp += f.v[2]; } else { rn += f.v[1]; rp += f.v[3]; }
    }
  };
  for (int k = 0; k <= NP + 1; ++k) {
    Pt P;
    point(L, k, Vint, P);
    const double ev[2] = {exp(-(P.V + P.offn) * L.iVt), exp((P.V + P.offp) * L.iVt)};
    double uc[2] = {0.0, 0.0};
    double R = 0.0, dRn = 0.0, dRp = 0.0;
    if (k >= 1 && k <= NP) {
      recomb(L, k, P.n, P.p, R, dRn, dRp);
      double rn, rp;
      ri_at(k, rn, rp);
      const double g = L.st(k, S_G) * L.gfrac;
      uc[0] = R + rn - g;
      uc[1] = R + rp - g;
    }
    rec(k, P_EVN) = ev[0]; rec(k, P_EVP) = ev[1];
    rec(k, P_DRN) = dRn; rec(k, P_DRP) = dRp;
    rec(k, P_N) = P.n; rec(k, P_P) = P.p;
    if (k <= NP) {
      const double dx = k < NP ? L.st(k, S_DX) : 0.0;
      const double wk = 0.5 * (dx_prev + dx);
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        if (k >= 1) iu[c] += 0.5 * dx_prev * (uc_prev[c] + uc[c]);
        const double mu = L.st(k, c == 0 ? S_MUN : S_MUP);
        sgl[c] += wk * ev[c] / mu;
        dbl[c] += wk * ev[c] * iu[c] / mu;
        uc_prev[c] = uc[c];
      }
      rec(k, P_IUN) = iu[0]; rec(k, P_IUP) = iu[1];
      dx_prev = dx;
    }
  }
  Pt P0, PR;
  point(L, 0, Vint, P0);
  point(L, NP + 1, Vint, PR);
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    const double sn = c == 0 ? -1.0 : 1.0;
    const double d0 = c == 0 ? P0.n : P0.p, dR = c == 0 ? PR.n : PR.p;
    const double e0 = exp(sn * ((c == 0 ? P0.offn : P0.offp) + P0.V) * L.iVt);
    const double eR = exp(sn * ((c == 0 ? PR.offn : PR.offp) + PR.V) * L.iVt);
    const double Bc = L.Vt * sn * (dR * eR - d0 * e0);
    a.lsc[(size_t)(L_SN + c) * a.Bp + l] = sgl[c];
    a.lsc[(size_t)(L_KN + c) * a.Bp + l] = (Bc - sn * dbl[c]) / sgl[c];
  }
}

// The interface traps of one edge beyond their steady occupation (`_interface_beyond`): per unit
// of (ln n_L, ln n_R, ln p_L, ln p_R) in the rates (`rate`), and the occupation's part in the
// four point rates and the charge (`dR`).
__device__ void iface_beyond(const Lane& L, int t, double nL, double nR, double pL, double pR,
                             cplx lap, double dt, cplx (&rate)[4], cplx (&crate)[4],
                             double (&dR)[5]) {
  const double Nt = L.itab(t, I_NT), Cn = L.itab(t, I_CN), Cp = L.itab(t, I_CP);
  const double nlo = L.itab(t, I_NT0LO), nhi = L.itab(t, I_NT0HI);
  const double plo = L.itab(t, I_PT0LO), phi = L.itab(t, I_PT0HI);
  const double iw = L.itab(t, I_IW), charge = L.itab(t, I_CHARGE);
  const double an = Cn * Nt, bp = Cp * Nt;
  double a = Cn * (nL + nR + nlo + nhi) + Cp * (pL + pR + plo + phi);
  const double b = Cn * (nL + nR) + Cp * (plo + phi);
  const double f = b / (a > 0.0 ? a : 1.0);
  dR[0] = -iw * an * (nL + nlo); dR[1] = -iw * an * (nR + nhi);
  dR[2] = iw * bp * (pL + plo);  dR[3] = iw * bp * (pR + phi);
  dR[4] = -charge * 0.5 * Nt * iw;
  const double da[4] = {Cn * nL, Cn * nR, Cp * pL, Cp * pR};
  const double db[4] = {Cn * nL, Cn * nR, 0.0, 0.0};
  if (!(Nt > 0.0)) a = 1.0;
  cplx hr, hc;
  transfer(a, lap, dt, hr, hc);
#pragma unroll
  for (int w = 0; w < 4; ++w) {
    rate[w] = ((db[w] - f * da[w]) / a) * hr;
    crate[w] = ((db[w] - f * da[w]) / a) * hc;
  }
  if (!(Nt > 0.0))
#pragma unroll
    for (int q = 0; q < 5; ++q) dR[q] = 0.0;
}

// The interface correction of row i's blocks: edges i-1 (this point its right end) and i (left).
__device__ void iface_rows(const Lane& L, int i, double Vint, cplx lap, double dt,
                           const double* rs, cplx (&dA)[3][3], cplx (&dB)[3][3],
                           cplx (&dC)[3][3]) {
  for (int side = 0; side < 2; ++side) {
    const int e = side == 0 ? i - 1 : i;  // the edge; this point is its right (0) or left (1) end
    if (e < 1 || e > L.NP - 1) continue;  // edges with both points interior
    const int t = (int)L.st(e, S_IFK);
    if (t < 0) continue;
    Pt p0, p1;
    point(L, e, Vint, p0);
    point(L, e + 1, Vint, p1);
    cplx rate_r[4], rate_c[4];
    double dR[5];
    iface_beyond(L, t, p0.n, p1.n, p0.p, p1.p, lap, dt, rate_r, rate_c, dR);
    const bool left_end = side == 1;
    const double rows[3] = {dR[4], left_end ? dR[0] : dR[1], left_end ? dR[2] : dR[3]};
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      // the charge (row 0) takes the occupation at a step's end, the rates its mean
      const cplx (&rate)[4] = r == 0 ? rate_c : rate_r;
      // own logarithms: this point's; other: the edge's other point's
      const cplx own_n = rate[left_end ? 0 : 1], own_p = rate[left_end ? 2 : 3];
      const cplx oth_n = rate[left_end ? 1 : 0], oth_p = rate[left_end ? 3 : 2];
      dB[r][1] = dB[r][1] + (rows[r] * rs[r]) * own_n;
      dB[r][2] = dB[r][2] + (rows[r] * rs[r]) * own_p;
      if (left_end) {  // coupling to the point after: C
        dC[r][1] = dC[r][1] + (rows[r] * rs[r]) * oth_n;
        dC[r][2] = dC[r][2] + (rows[r] * rs[r]) * oth_p;
      } else {  // to the point before: A
        dA[r][1] = dA[r][1] + (rows[r] * rs[r]) * oth_n;
        dA[r][2] = dA[r][2] + (rows[r] * rs[r]) * oth_p;
      }
    }
  }
}

__device__ void inv3c(const cplx (&M)[3][3], cplx (&Mi)[3][3]) {
  const cplx c00 = M[1][1] * M[2][2] - M[1][2] * M[2][1];
  const cplx c01 = M[0][2] * M[2][1] - M[0][1] * M[2][2];
  const cplx c02 = M[0][1] * M[1][2] - M[0][2] * M[1][1];
  const cplx c10 = M[1][2] * M[2][0] - M[1][0] * M[2][2];
  const cplx c11 = M[0][0] * M[2][2] - M[0][2] * M[2][0];
  const cplx c12 = M[0][2] * M[1][0] - M[0][0] * M[1][2];
  const cplx c20 = M[1][0] * M[2][1] - M[1][1] * M[2][0];
  const cplx c21 = M[0][1] * M[2][0] - M[0][0] * M[2][1];
  const cplx c22 = M[0][0] * M[1][1] - M[0][1] * M[1][0];
  const cplx idet = mk(1.0) / (M[0][0] * c00 + M[0][1] * c10 + M[0][2] * c20);
  Mi[0][0] = c00 * idet; Mi[0][1] = c01 * idet; Mi[0][2] = c02 * idet;
  Mi[1][0] = c10 * idet; Mi[1][1] = c11 * idet; Mi[1][2] = c12 * idet;
  Mi[2][0] = c20 * idet; Mi[2][1] = c21 * idet; Mi[2][2] = c22 * idet;
}

// The interface recombination's tangent of point k (edges k-1 and k): the steady occupation's
// derivatives in the points' logarithms and the traps' extra rates (`_interface_rates`).
__device__ void iface_tangent(const Lane& L, int k, double Vint, cplx lap, double dt,
                              const cplx (&dlnn)[3], const cplx (&dlnp)[3], cplx& tn, cplx& tp) {
  tn = mk(0.0); tp = mk(0.0);
  for (int e = k - 1; e <= k; ++e) {
    if (e < 0 || e > L.NP) continue;
    const int t = (int)L.st(e, S_IFK);
    if (t < 0) continue;
    Pt p0, p1;
    point(L, e, Vint, p0);
    point(L, e + 1, Vint, p1);
    Iface f;
    iface_edge(L, t, p0.n, p1.n, p0.p, p1.p, f, true);
    // this edge's two points in dlnn/dlnp's frame: index 0 is k-1, 1 is k, 2 is k+1
    const int j0 = e - (k - 1), j1 = j0 + 1;
    const cplx v[4] = {dlnn[j0], dlnn[j1], dlnp[j0], dlnp[j1]};
    const int qn = e == k ? 0 : 1, qp = e == k ? 2 : 3;  // this point's left or right rates
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      tn = tn + f.d[w][qn] * v[w];
      tp = tp + f.d[w][qp] * v[w];
    }
    // beyond the steady occupation (only edges with both points interior move, as jaxdd's)
    cplx rate[4], crate[4];
    double dR[5];
    iface_beyond(L, t, p0.n, p1.n, p0.p, p1.p, lap, dt, rate, crate, dR);
    cplx df = mk(0.0);
#pragma unroll
    for (int w = 0; w < 4; ++w) df = df + rate[w] * v[w];
    tn = tn + dR[qn] * df;
    tp = tp + dR[qp] * df;
  }
}

__global__ void __launch_bounds__(64) admittance_kernel(Args a) {
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < (long)a.Bp * a.nf;
       t += (long)gridDim.x * blockDim.x) {
    const int l = (int)(t % a.Bp), q = (int)(t / a.Bp);
    if (l >= a.B) continue;
    Lane L;
    lane_init(L, a, l);
    const int NP = L.NP;
    const double Vint = a.vint[l];
    const cplx lap = mk(a.laps[2 * q], a.laps[2 * q + 1]);
    const long slot = (long)blockIdx.x * blockDim.x + threadIdx.x;
    auto rec = [&](int k, int f) { return a.rec[((size_t)k * P_WORDS + f) * a.Bp + l]; };
    auto scr = [&](int k, int f) -> double& { return a.scr[((size_t)k * W_WORDS + f) * a.T + slot]; };
    const double e = L.left();
    // ---- forward elimination of (J + iw M + traps) dy = -dF/dV
    cplx cp[3][3], dp[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) { dp[r] = mk(0.0); for (int c = 0; c < 3; ++c) cp[r][c] = mk(0.0); }
    for (int i = 1; i <= NP; ++i) {
      cplx A[3][3], Bm[3][3], Cm[3][3];
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          A[r][c] = mk(rec(i, P_A + 3 * r + c));
          Bm[r][c] = mk(rec(i, P_B + 3 * r + c));
          Cm[r][c] = mk(rec(i, P_C + 3 * r + c));
        }
      Bm[1][1] = Bm[1][1] + rec(i, P_MN) * lap;
      Bm[2][2] = Bm[2][2] + rec(i, P_MP) * lap;
      // bulk traps beyond their instantaneous occupation
      const double ta = rec(i, P_TA);
      cplx h, hc_unused;
      transfer(ta, lap, a.dt, h, hc_unused);  // neutral levels: the rates only
      const double fsc = L.st(i, S_FAC) * L.st(i, S_SC);
      const cplx rn = (rec(i, P_TDN) / ta) * h, rp = (rec(i, P_TDP) / ta) * h;
      Bm[1][1] = Bm[1][1] - (fsc * rec(i, P_TRN)) * rn;
      Bm[1][2] = Bm[1][2] - (fsc * rec(i, P_TRN)) * rp;
      Bm[2][1] = Bm[2][1] - (fsc * rec(i, P_TRP)) * rn;
      Bm[2][2] = Bm[2][2] - (fsc * rec(i, P_TRP)) * rp;
      if ((int)L.st(i - 1, S_IFK) >= 0 || (int)L.st(i, S_IFK) >= 0) {
        const double rs[3] = {Q * L.st(i, S_SP), -L.st(i, S_FAC) * L.st(i, S_SC),
                              -L.st(i, S_FAC) * L.st(i, S_SC)};
        iface_rows(L, i, Vint, lap, a.dt, rs, A, Bm, Cm);
      }
      // the drive: the residual's derivative in V_int (the contacts' potentials)
      cplx r[3] = {mk(0.0), mk(0.0), mk(0.0)};
      if (i == 1)
#pragma unroll
        for (int c = 0; c < 3; ++c) r[c] = r[c] - mk(rec(1, P_A + 3 * c) * 0.5 * e);
      if (i == NP)
#pragma unroll
        for (int c = 0; c < 3; ++c) r[c] = r[c] - mk(rec(NP, P_C + 3 * c) * (-0.5 * e));
      cplx M[3][3], Mi[3][3];
#pragma unroll
      for (int rr = 0; rr < 3; ++rr)
#pragma unroll
        for (int c = 0; c < 3; ++c)
          M[rr][c] = Bm[rr][c] - (A[rr][0] * cp[0][c] + A[rr][1] * cp[1][c] + A[rr][2] * cp[2][c]);
      inv3c(M, Mi);
      cplx t3[3];
#pragma unroll
      for (int rr = 0; rr < 3; ++rr)
        t3[rr] = r[rr] - (A[rr][0] * dp[0] + A[rr][1] * dp[1] + A[rr][2] * dp[2]);
#pragma unroll
      for (int rr = 0; rr < 3; ++rr) {
        dp[rr] = Mi[rr][0] * t3[0] + Mi[rr][1] * t3[1] + Mi[rr][2] * t3[2];
#pragma unroll
        for (int c = 0; c < 3; ++c)
          cp[rr][c] = Mi[rr][0] * Cm[0][c] + Mi[rr][1] * Cm[1][c] + Mi[rr][2] * Cm[2][c];
      }
#pragma unroll
      for (int rr = 0; rr < 3; ++rr) {
        scr(i, W_D + 2 * rr) = dp[rr].re; scr(i, W_D + 2 * rr + 1) = dp[rr].im;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          scr(i, W_C + 2 * (3 * rr + c)) = cp[rr][c].re;
          scr(i, W_C + 2 * (3 * rr + c) + 1) = cp[rr][c].im;
        }
      }
    }
    // ---- back substitution: dy_i = d'_i - c'_i dy_{i+1}
    cplx x[3] = {mk(0.0), mk(0.0), mk(0.0)};
    for (int i = NP; i >= 1; --i) {
      cplx nx[3];
#pragma unroll
      for (int rr = 0; rr < 3; ++rr) {
        cplx v = mk(scr(i, W_D + 2 * rr), scr(i, W_D + 2 * rr + 1));
#pragma unroll
        for (int c = 0; c < 3; ++c)
          v = v - mk(scr(i, W_C + 2 * (3 * rr + c)), scr(i, W_C + 2 * (3 * rr + c) + 1)) * x[c];
        nx[rr] = v;
      }
#pragma unroll
      for (int rr = 0; rr < 3; ++rr) {
        x[rr] = nx[rr];
        scr(i, W_D + 2 * rr) = nx[rr].re; scr(i, W_D + 2 * rr + 1) = nx[rr].im;
      }
    }
    // ---- the current's tangent, left to right: base (dt-free, the traps' extra rates in it)
    // and per-dt parts for both carriers, and the displacement current
    auto dyv = [&](int k, int c) -> cplx {
      if (k < 1 || k > NP) return mk(0.0);
      return mk(scr(k, W_D + 2 * c), scr(k, W_D + 2 * c + 1));
    };
    auto dV = [&](int k) -> cplx {
      if (k == 0) return mk(0.5 * e);
      if (k == NP + 1) return mk(-0.5 * e);
      return dyv(k, 0);
    };
    const double sign = -L.left();
    const double Vt = L.Vt;
    cplx dsgl[2] = {mk(0.0), mk(0.0)}, ddb_b[2] = {mk(0.0), mk(0.0)}, ddb_t[2] = {mk(0.0), mk(0.0)};
    cplx diu_b[2] = {mk(0.0), mk(0.0)}, diu_t[2] = {mk(0.0), mk(0.0)};
    cplx dS_b[2] = {mk(0.0), mk(0.0)}, dS_t[2] = {mk(0.0), mk(0.0)};
    cplx sumJ_b[2] = {mk(0.0), mk(0.0)}, sumJ_t[2] = {mk(0.0), mk(0.0)};
    cplx duc_prev_b[2] = {mk(0.0), mk(0.0)}, duc_prev_t[2] = {mk(0.0), mk(0.0)};
    cplx dJD = mk(0.0);
    double hsum = 0.0, dx_prev = 0.0, h_prev = 0.0;
    // `currDiffInt = 1`: each interval's Scharfetter-Gummel flux instead of the integral form
    // (jaxdd batch.py:366-369), its tangent from the points at both ends of the interval
    const bool cdiff = L.sc(C_CURRDIFF) > 0.0;
    cplx jd_prev[2] = {mk(0.0), mk(0.0)};
    Pt Pa, Pb;
    if (cdiff) point(L, 0, Vint, Pa);
    for (int k = 0; k <= NP; ++k) {
      const double hk = L.st(k, S_H);
      const double dx = k < NP ? L.st(k, S_DX) : 0.0;
      const double wk = 0.5 * (dx_prev + dx);
      const double width = k == 0 ? hk : 0.5 * (h_prev + hk);
      hsum += hk;
      // the interface recombination's tangent at k and k+1 (through term)
      cplx dRi_k[2] = {mk(0.0), mk(0.0)}, dRi_k1[2] = {mk(0.0), mk(0.0)};
      // points k and k + 1 touch edges k - 1 .. k + 1
      bool trapped = false;
      for (int ee = k - 1; ee <= k + 1; ++ee)
        if (ee >= 0 && ee <= NP && (int)L.st(ee, S_IFK) >= 0) trapped = true;
      if (trapped) {
        const cplx ln[3] = {dyv(k - 1, 1), dyv(k, 1), dyv(k + 1, 1)};
        const cplx lp[3] = {dyv(k - 1, 2), dyv(k, 2), dyv(k + 1, 2)};
        iface_tangent(L, k, Vint, lap, a.dt, ln, lp, dRi_k[0], dRi_k[1]);
        if (k + 1 <= NP + 1) {
          const cplx ln1[3] = {dyv(k, 1), dyv(k + 1, 1), dyv(k + 2, 1)};
          const cplx lp1[3] = {dyv(k, 2), dyv(k + 1, 2), dyv(k + 2, 2)};
          iface_tangent(L, k + 1, Vint, lap, a.dt, ln1, lp1, dRi_k1[0], dRi_k1[1]);
        }
      }
      // the bulk traps' extra rates at k
      cplx dU[2] = {mk(0.0), mk(0.0)};
      if (k >= 1) {
        const double ta = rec(k, P_TA);
        cplx h, hc_unused;
        transfer(ta, lap, a.dt, h, hc_unused);
        const cplx df = ((rec(k, P_TDN) / ta) * h) * dyv(k, 1) + ((rec(k, P_TDP) / ta) * h) * dyv(k, 2);
        dU[0] = rec(k, P_TRN) * df;
        dU[1] = rec(k, P_TRP) * df;
      }
      const bool iface_k = L.st(k, S_IFK) > -1.5;
      if (cdiff) point(L, k + 1, Vint, Pb);
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const double sn = c == 0 ? -1.0 : 1.0;
        const double ev = rec(k, c == 0 ? P_EVN : P_EVP), iu = rec(k, c == 0 ? P_IUN : P_IUP);
        const double mu = L.st(k, c == 0 ? S_MUN : S_MUP);
        const cplx dev = (ev * sn / Vt) * dV(k);
        cplx duc_b = mk(0.0), duc_t = mk(0.0);
        if (k >= 1) {
          duc_b = rec(k, P_DRN) * dyv(k, 1) + rec(k, P_DRP) * dyv(k, 2) + dRi_k[c] + dU[c];
          duc_t = rec(k, c == 0 ? P_N : P_P) * dyv(k, 1 + c);
          diu_b[c] = diu_b[c] + (0.5 * dx_prev) * (duc_prev_b[c] + duc_b);
          diu_t[c] = diu_t[c] + (0.5 * dx_prev) * (duc_prev_t[c] + duc_t);
        }
        dsgl[c] = dsgl[c] + (wk / mu) * dev;
        ddb_b[c] = ddb_b[c] + (wk * iu / mu) * dev + (wk * ev / mu) * diu_b[c];
        ddb_t[c] = ddb_t[c] + (wk * ev / mu) * diu_t[c];
        const cplx dS_prev_b = dS_b[c], dS_prev_t = dS_t[c];
        if (k >= 1) {
          dS_b[c] = dS_b[c] + (sn * Q * L.L * width) * duc_b;
          dS_t[c] = dS_t[c] + (sn * Q * L.L * width) * duc_t;
        }
        const cplx thr = (sn * 0.5 * Q * L.L * hk) * (dRi_k[c] + dRi_k1[c]);
        if (cdiff) {
          // d[sn q mu V_T (d1 B(-x) - d0 B(x))]/(L h), x = sn (Vg1 - Vg0)/V_T; across an
          // interface the interval before it plus the current through its traps
          const double d0 = c == 0 ? Pa.n : Pa.p, d1 = c == 0 ? Pb.n : Pb.p;
          const double g0 = Pa.V + (c == 0 ? Pa.offn : Pa.offp);
          const double g1 = Pb.V + (c == 0 ? Pb.offn : Pb.offp);
          double bf, bb, dbf, dbb;
          bern_pair(sn * (g1 - g0) / Vt, L.simss, bf, bb, dbf, dbb);
          const cplx dxk = (sn / Vt) * (dV(k + 1) - dV(k));
          const cplx djd = (sn * Q * mu * Vt / (L.L * hk)) *
                           (d1 * (bb * dyv(k + 1, 1 + c) - dbb * dxk) -
                            d0 * (bf * dyv(k, 1 + c) + dbf * dxk));
          sumJ_b[c] = sumJ_b[c] + hk * (iface_k ? jd_prev[c] + thr : djd);
          jd_prev[c] = djd;
        } else if (iface_k) {
          sumJ_b[c] = sumJ_b[c] + hk * (dS_prev_b + thr);
          sumJ_t[c] = sumJ_t[c] + hk * dS_prev_t;
        } else {
          sumJ_b[c] = sumJ_b[c] + hk * dS_b[c];
          sumJ_t[c] = sumJ_t[c] + hk * dS_t[c];
        }
        duc_prev_b[c] = duc_b;
        duc_prev_t[c] = duc_t;
      }
      // the displacement current on interval k (its per-dt part)
      const double epsk = a.eps[(size_t)k * a.Bp + l];
      dJD = dJD + (hk * sign * epsk / (L.L * hk)) * (dV(k + 1) - dV(k));
      dx_prev = dx;
      h_prev = hk;
      if (cdiff) Pa = Pb;
    }
    // K's tangent and the total
    cplx Yb = mk(0.0), Yt = mk(0.0);
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const double sn = c == 0 ? -1.0 : 1.0;
      const double sgl = a.lsc[(size_t)(L_SN + c) * a.Bp + l], Kc = a.lsc[(size_t)(L_KN + c) * a.Bp + l];
      // the contacts' densities are fixed; their exp(sn Vg / V_T) move with the voltage
      Pt P0, PR;
      point(L, 0, Vint, P0);
      point(L, NP + 1, Vint, PR);
      const double d0 = c == 0 ? P0.n : P0.p, dR = c == 0 ? PR.n : PR.p;
      const double e0 = exp(sn * ((c == 0 ? P0.offn : P0.offp) + P0.V) / Vt);
      const double eR = exp(sn * ((c == 0 ? PR.offn : PR.offp) + PR.V) / Vt);
      const cplx dBc = (Vt * sn) * ((dR * eR * sn / Vt) * dV(NP + 1) - (d0 * e0 * sn / Vt) * dV(0));
      const cplx dK_b = (1.0 / sgl) * (dBc - sn * ddb_b[c]) - (Kc / sgl) * dsgl[c];
      const cplx dK_t = (-sn / sgl) * ddb_t[c];
      if (!cdiff) {  // the differential current has no K
        Yb = Yb + sign * (Q * hsum) * dK_b;
        Yt = Yt + sign * (Q * hsum) * dK_t;
      }
      Yb = Yb + sign * sumJ_b[c];
      Yt = Yt + sign * sumJ_t[c];
    }
    Yt = Yt + dJD;
    const cplx Y = (1.0 / hsum) * (Yb + lap * Yt);
    a.Y[((size_t)q * 2) * a.Bp + l] = Y.re;
    a.Y[((size_t)q * 2 + 1) * a.Bp + l] = Y.im;
  }
}

// ------------------------------------------------------------------------------------ ions
//
// With mobile ions (jaxdd `_admittance` with `ions`, impedance.py:242-353) the ions are unknowns
// of their own: the 5x5 blocks of a time step of dti = 1 from the steady state (the traps at
// their steady occupation, `_time_terms` without occupations), `B + (iw - 1) M` on the diagonal,
// the bulk and interface traps' blocks on the carriers' 3x3, and the ion slots as a border that
// keeps each region's number (`_ion_constraints_time`); the current of a time step, linearised,
// gains each region's ion current (`_ion_currents`, batch.py:421-483).

// Per node of the ions' record, [node][word][lane]: the 5x5 blocks, the mass, the slot columns
// U (anion row, cation row), the constraints' border W (at ln a, at ln c), and the ions'
// densities and exp(-+V/V_T) of the steady state.
enum { R_A = 0, R_B = 25, R_C = 50, R_M = 75, R_U3 = 80, R_U4, R_W3, R_W4, R_NA, R_NC, R_EVA,
       R_EVC, R5_WORDS };
// At a contact (nodes 0 and np+1, whose rows' words are free) where an ion region reaches it,
// per species (anion, cation): its ln density from its neighbour's, `_ion_full`'s at a step
// (dti = 1: ln(B(x)/B(-x))) and Boltzmann's (dti = 0); d(ln density)/d(V of the neighbour) of
// the first; and the region's number's derivative in the neighbour's potential through it.
enum { CT_LNR = R_A, CT_SR = R_A + 2, CT_LNB = R_A + 4, CT_WV = R_A + 6, CT_WORDS = 8 };
// Per node of a (device, frequency) thread: c' (25 complex) and [-dF | U_0 .. U_K-1] (5 (1 + K)
// complex; each slot's column, anion slots first).
enum { V_C = 0, V_D = 50 };
__host__ __device__ constexpr int vwords(int K) { return V_D + 10 * (1 + K); }

struct IonArgs {
  const double* X;           // [np+2][DD_NT][Bp]: permittivity, anion and cation mobility
  const double* state_logs;  // [DD_MAXK][Bp]
  double* rec5;              // [np+2][R5_WORDS][Bp]
  double* scr5;              // [np+2][V_WORDS][T]
};

// A point of the steady state with its ions' logarithms (their Boltzmann profiles).
__device__ void ion_point(const tr::View& W, int k, double Vint, const double* logs, tr::TP& P) {
  const Lane& L = W.L;
  if (k == 0 || k == L.NP + 1) contact(L, k != 0, Vint, P.c);
  else { P.c.V = *L.y(0, k, 0); P.c.lnn = *L.y(0, k, 1); P.c.lnp = *L.y(0, k, 2); }
  P.c.n = exp(P.c.lnn);
  P.c.p = exp(P.c.lnp);
  P.c.offn = L.st(k, S_OFFN);
  P.c.offp = L.st(k, S_OFFP);
  P.c.sl = slots_at(L, k);
  const bool inner = k >= 1 && k <= L.NP;
  P.la = inner && P.c.sl.a >= 0 ? logs[P.c.sl.a] + P.c.V * L.iVt : 0.0;
  P.lc = inner && P.c.sl.c >= 0 ? logs[L.ka + P.c.sl.c] - P.c.V * L.iVt : 0.0;
  P.a = exp(P.la);
  P.c2 = exp(P.lc);
  P.c.da = P.c.sl.a >= 0 ? P.a : 0.0;
  P.c.dc = P.c.sl.c >= 0 ? P.c2 : 0.0;
}

__device__ void ion_view(tr::View& W, const Args& a, const IonArgs& b, int l) {
  lane_init(W.L, a, l);
  for (int k = 0; k < DD_MAXK; ++k) W.L.tot[k] = k < a.K ? W.L.sc(C_TOT0 + k) : 0.0;
  W.X = b.X;
  W.Yb = nullptr;
  W.ybuf = 0;
  W.simss = a.simss;
  W.zimt = 0;
  W.BD = nullptr;
}

// The ions' record of each device: its rows as a step of dti = 1 from the steady state itself.
template <int K>
__global__ void __launch_bounds__(32) prepare_ions_kernel(Args a, IonArgs b) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= a.B) return;
  tr::View W;
  ion_view(W, a, b, l);
  const Lane& L = W.L;
  const int NP = L.NP;
  const double Vint = a.vint[l];
  double logs[K], zero[K];
#pragma unroll
  for (int k = 0; k < K; ++k) { logs[k] = b.state_logs[(size_t)k * a.Bp + l]; zero[k] = 0.0; }
  auto rec = [&](int k, int f) -> double& {
    return b.rec5[((size_t)k * R5_WORDS + f) * a.Bp + l];
  };
  tr::TP pm, pc, pn;
  ion_point(W, 0, Vint, logs, pm);
  ion_point(W, 1, Vint, logs, pc);
  Flux el, er;
  flux(L, pm.c, pc.c, L.st(0, S_MUN), L.st(0, S_MUP), el);
  for (int i = 1; i <= NP; ++i) {
    ion_point(W, i + 1, Vint, logs, pn);
    flux(L, pc.c, pn.c, L.st(i, S_MUN), L.st(i, S_MUP), er);
    double A[5][5], Bm[5][5], Cm[5][5], r[5], U[5][K], M[5];
    tr::row5<K, true>(W, i, pm, pc, pn, el, er, L.st(i - 1, S_H), L.st(i, S_H),
                      (int)L.st(i - 1, S_IFK), (int)L.st(i, S_IFK), 1.0, 0.0, 0.0, 0.0, pc.c.n,
                      pc.c.p, pc.c.da, pc.c.dc, zero, A, Bm, Cm, r, U, M);
#pragma unroll
    for (int rr = 0; rr < 5; ++rr) {
#pragma unroll
      for (int c = 0; c < 5; ++c) {
        rec(i, R_A + 5 * rr + c) = A[rr][c];
        rec(i, R_B + 5 * rr + c) = Bm[rr][c];
        rec(i, R_C + 5 * rr + c) = Cm[rr][c];
      }
      rec(i, R_M + rr) = M[rr];
    }
    rec(i, R_U3) = pc.c.sl.a >= 0 ? pick<K>(U[3], pc.c.sl.a) : 0.0;
    rec(i, R_U4) = pc.c.sl.c >= 0 ? pick<K>(U[4], L.ka + pc.c.sl.c) : 0.0;
    // the constraints' border: each region's number in its points' ion logarithms
    const double hLm = L.st(i - 1, S_H) * L.L, hLp = L.st(i, S_H) * L.L;
    double w3 = 0.0, w4 = 0.0;
    if (pc.c.sl.a >= 0 && L.tot[pc.c.sl.a] > 0.0)
      w3 = 0.5 * ((pm.c.sl.a == pc.c.sl.a ? hLm : 0.0) + (pn.c.sl.a == pc.c.sl.a ? hLp : 0.0)) *
           pc.a / L.tot[pc.c.sl.a];
    const int kc = L.ka + pc.c.sl.c;
    if (pc.c.sl.c >= 0 && L.tot[kc] > 0.0)
      w4 = 0.5 * ((pm.c.sl.c == pc.c.sl.c ? hLm : 0.0) + (pn.c.sl.c == pc.c.sl.c ? hLp : 0.0)) *
           pc.c2 / L.tot[kc];
    rec(i, R_W3) = w3;
    rec(i, R_W4) = w4;
    pm = pc; pc = pn; el = er;
  }
  for (int k = 0; k <= NP + 1; ++k) {
    tr::TP P;
    ion_point(W, k, Vint, logs, P);
    rec(k, R_NA) = P.c.da;
    rec(k, R_NC) = P.c.dc;
    rec(k, R_EVA) = exp(-P.c.V * L.iVt);
    rec(k, R_EVC) = exp(P.c.V * L.iVt);
  }
  // the contacts that an ion region reaches (`_ion_full`, solver.py:1315-1346): no flux over
  // the contact's interval at a step, Boltzmann's in the steady state; the region's number
  // (trapezoidal over its intervals, `_ion_constraints_time`) takes the contact's share
  for (int side = 0; side < 2; ++side) {
    const int c = side == 0 ? 0 : NP + 1, nb = side == 0 ? 1 : NP;
    tr::TP Pc, Pn;
    ion_point(W, c, Vint, logs, Pc);
    ion_point(W, nb, Vint, logs, Pn);
    const double x = side == 0 ? (Pn.c.V - Pc.c.V) * L.iVt : (Pc.c.V - Pn.c.V) * L.iVt;
    double bf, bb, dbf, dbb;
    bern_pair(x, L.simss, bf, bb, dbf, dbb);
    const double r = log(bf) - log(bb), dr = dbf / bf + dbb / bb;
    const double hL = L.st(side == 0 ? 0 : NP, S_H) * L.L;
#pragma unroll
    for (int sp = 0; sp < 2; ++sp) {
      const int reg = sp == 0 ? Pc.c.sl.a : Pc.c.sl.c;
      const int regn = sp == 0 ? Pn.c.sl.a : Pn.c.sl.c;
      const int q = sp == 0 ? reg : L.ka + reg;
      double lnR = 0.0, sR = 0.0, lnB = 0.0, wv = 0.0;
      if (reg >= 0) {
        const double lnn = sp == 0 ? Pn.la : Pn.lc;
        // anions: ln a_0 = ln a_1 + r(x), ln a_N+1 = ln a_N - r(x); the cations the other way
        const double sg = (sp == 0) == (side == 0) ? 1.0 : -1.0;
        lnR = lnn + sg * r;
        sR = (sp == 0 ? 1.0 : -1.0) * dr * L.iVt;
        lnB = lnn + (sp == 0 ? 1.0 : -1.0) * (Pc.c.V - Pn.c.V) * L.iVt;
        const double tq = pick<K>(L.tot, q);
        if (regn == reg && tq > 0.0) {
          const double w = 0.5 * hL * exp(lnR) / tq;
          rec(nb, sp == 0 ? R_W3 : R_W4) += w;
          wv = w * sR;
        }
      }
      rec(c, CT_LNR + sp) = lnR;
      rec(c, CT_SR + sp) = sR;
      rec(c, CT_LNB + sp) = lnB;
      rec(c, CT_WV + sp) = wv;
    }
  }
}

// M^-1 applied in place, M = [[P, Q], [R, S]] complex, by its partition (as `tr::partition`).
struct CPart {
  cplx Pi[3][3], PiQ[3][2], R[2][3], Si[2][2];
};

__device__ void cpartition(const cplx (&M)[5][5], CPart& f) {
  cplx P[3][3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) P[r][c] = M[r][c];
  inv3c(P, f.Pi);
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 2; ++c)
      f.PiQ[r][c] = f.Pi[r][0] * M[0][3 + c] + f.Pi[r][1] * M[1][3 + c] + f.Pi[r][2] * M[2][3 + c];
  cplx S[2][2];
#pragma unroll
  for (int r = 0; r < 2; ++r) {
#pragma unroll
    for (int c = 0; c < 3; ++c) f.R[r][c] = M[3 + r][c];
#pragma unroll
    for (int c = 0; c < 2; ++c)
      S[r][c] = M[3 + r][3 + c] - (M[3 + r][0] * f.PiQ[0][c] + M[3 + r][1] * f.PiQ[1][c] +
                                   M[3 + r][2] * f.PiQ[2][c]);
  }
  const cplx idet = mk(1.0) / (S[0][0] * S[1][1] - S[0][1] * S[1][0]);
  f.Si[0][0] = S[1][1] * idet; f.Si[0][1] = mk(0.0) - S[0][1] * idet;
  f.Si[1][0] = mk(0.0) - S[1][0] * idet; f.Si[1][1] = S[0][0] * idet;
}

__device__ void capply(const CPart& f, cplx (&v)[5]) {
  cplx yt[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) yt[r] = f.Pi[r][0] * v[0] + f.Pi[r][1] * v[1] + f.Pi[r][2] * v[2];
  cplx w[2];
#pragma unroll
  for (int r = 0; r < 2; ++r)
    w[r] = v[3 + r] - (f.R[r][0] * yt[0] + f.R[r][1] * yt[1] + f.R[r][2] * yt[2]);
  const cplx z0 = f.Si[0][0] * w[0] + f.Si[0][1] * w[1];
  const cplx z1 = f.Si[1][0] * w[0] + f.Si[1][1] * w[1];
#pragma unroll
  for (int r = 0; r < 3; ++r) v[r] = yt[r] - (f.PiQ[r][0] * z0 + f.PiQ[r][1] * z1);
  v[3] = z0;
  v[4] = z1;
}

// The K x K system M z = r (complex) by Gauss-Jordan elimination with partial pivoting, z over r.
template <int K>
__device__ void csolve(cplx (&M)[K][K], cplx (&r)[K]) {
  for (int c = 0; c < K; ++c) {
    int piv = c;
    double best = M[c][c].re * M[c][c].re + M[c][c].im * M[c][c].im;
    for (int rr = c + 1; rr < K; ++rr) {
      const double v = M[rr][c].re * M[rr][c].re + M[rr][c].im * M[rr][c].im;
      if (v > best) { best = v; piv = rr; }
    }
    if (piv != c) {
      for (int q = 0; q < K; ++q) { const cplx t = M[c][q]; M[c][q] = M[piv][q]; M[piv][q] = t; }
      const cplx t = r[c]; r[c] = r[piv]; r[piv] = t;
    }
    const cplx inv = mk(1.0) / M[c][c];
    for (int q = 0; q < K; ++q) M[c][q] = M[c][q] * inv;
    r[c] = r[c] * inv;
    for (int rr = 0; rr < K; ++rr) {
      if (rr == c) continue;
      const cplx f = M[rr][c];
      for (int q = 0; q < K; ++q) M[rr][q] = M[rr][q] - f * M[c][q];
      r[rr] = r[rr] - f * r[c];
    }
  }
}

template <int K>
__global__ void __launch_bounds__(64) admittance_ions_kernel(Args a, IonArgs b) {
  constexpr int NC = 1 + K, VW = vwords(K);
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < (long)a.Bp * a.nf;
       t += (long)gridDim.x * blockDim.x) {
    const int l = (int)(t % a.Bp), q = (int)(t / a.Bp);
    if (l >= a.B) continue;
    tr::View W;
    ion_view(W, a, b, l);
    const Lane& L = W.L;
    const int NP = L.NP;
    const double Vint = a.vint[l];
    const cplx lap = mk(a.laps[2 * q], a.laps[2 * q + 1]);
    const long slot = (long)blockIdx.x * blockDim.x + threadIdx.x;
    auto rec = [&](int k, int f) { return a.rec[((size_t)k * P_WORDS + f) * a.Bp + l]; };
    auto r5 = [&](int k, int f) { return b.rec5[((size_t)k * R5_WORDS + f) * a.Bp + l]; };
    auto scr = [&](int k, int f) -> double& {
      return b.scr5[((size_t)k * VW + f) * a.T + slot];
    };
    const double e = L.left();
    // ---- forward elimination of (J + (iw - 1) M + traps) [dy | X_U] = [-dF/dV | U]
    cplx cp[5][5], dp[5][NC];
#pragma unroll
    for (int rr = 0; rr < 5; ++rr) {
#pragma unroll
      for (int c = 0; c < 5; ++c) cp[rr][c] = mk(0.0);
#pragma unroll
      for (int c = 0; c < NC; ++c) dp[rr][c] = mk(0.0);
    }
    for (int i = 1; i <= NP; ++i) {
      cplx A[5][5], Bm[5][5], Cm[5][5];
#pragma unroll
      for (int rr = 0; rr < 5; ++rr)
#pragma unroll
        for (int c = 0; c < 5; ++c) {
          A[rr][c] = mk(r5(i, R_A + 5 * rr + c));
          Bm[rr][c] = mk(r5(i, R_B + 5 * rr + c));
          Cm[rr][c] = mk(r5(i, R_C + 5 * rr + c));
        }
      const cplx lm1 = lap - mk(1.0);  // the step's dti = 1 is in B already
#pragma unroll
      for (int rr = 0; rr < 5; ++rr) Bm[rr][rr] = Bm[rr][rr] + r5(i, R_M + rr) * lm1;
      // bulk traps beyond their instantaneous occupation (the carriers' 3x3)
      const double ta = rec(i, P_TA);
      cplx h, hc_unused;
      transfer(ta, lap, a.dt, h, hc_unused);  // neutral levels: the rates only
      const double fsc = L.st(i, S_FAC) * L.st(i, S_SC);
      const cplx rn = (rec(i, P_TDN) / ta) * h, rp = (rec(i, P_TDP) / ta) * h;
      Bm[1][1] = Bm[1][1] - (fsc * rec(i, P_TRN)) * rn;
      Bm[1][2] = Bm[1][2] - (fsc * rec(i, P_TRN)) * rp;
      Bm[2][1] = Bm[2][1] - (fsc * rec(i, P_TRP)) * rn;
      Bm[2][2] = Bm[2][2] - (fsc * rec(i, P_TRP)) * rp;
      if ((int)L.st(i - 1, S_IFK) >= 0 || (int)L.st(i, S_IFK) >= 0) {
        const double rs[3] = {Q * L.st(i, S_SP), -L.st(i, S_FAC) * L.st(i, S_SC),
                              -L.st(i, S_FAC) * L.st(i, S_SC)};
        cplx dA[3][3], dB[3][3], dC[3][3];
#pragma unroll
        for (int rr = 0; rr < 3; ++rr)
#pragma unroll
          for (int c = 0; c < 3; ++c) { dA[rr][c] = mk(0.0); dB[rr][c] = mk(0.0); dC[rr][c] = mk(0.0); }
        iface_rows(L, i, Vint, lap, a.dt, rs, dA, dB, dC);
#pragma unroll
        for (int rr = 0; rr < 3; ++rr)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            A[rr][c] = A[rr][c] + dA[rr][c];
            Bm[rr][c] = Bm[rr][c] + dB[rr][c];
            Cm[rr][c] = Cm[rr][c] + dC[rr][c];
          }
      }
      // right-hand sides: -dF/dV (the contacts' potentials), then the slots' columns (the
      // point's anion slot in the anions' row, its cation slot in the cations')
      const Slots si = slots_at(L, i);
      const int ja = si.a >= 0 ? si.a : -1, jc = si.c >= 0 ? L.ka + si.c : -1;
      const double u3 = r5(i, R_U3), u4 = r5(i, R_U4);
      cplx rhs[5][NC];
#pragma unroll
      for (int rr = 0; rr < 5; ++rr) {
        double dF = 0.0;
        if (i == 1) dF += r5(1, R_A + 5 * rr) * 0.5 * e;
        if (i == NP) dF += r5(NP, R_C + 5 * rr) * (-0.5 * e);
        rhs[rr][0] = mk(-dF);
#pragma unroll
        for (int c = 1; c < NC; ++c)
          rhs[rr][c] = mk(rr == 3 && c - 1 == ja ? u3 : rr == 4 && c - 1 == jc ? u4 : 0.0);
      }
      cplx M[5][5];
#pragma unroll
      for (int rr = 0; rr < 5; ++rr) {
#pragma unroll
        for (int c = 0; c < 5; ++c) {
          cplx s = Bm[rr][c];
#pragma unroll
          for (int k = 0; k < 5; ++k) s = s - A[rr][k] * cp[k][c];
          M[rr][c] = s;
        }
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          cplx s = rhs[rr][c];
#pragma unroll
          for (int k = 0; k < 5; ++k) s = s - A[rr][k] * dp[k][c];
          rhs[rr][c] = s;
        }
      }
      CPart f;
      cpartition(M, f);
#pragma unroll
      for (int c = 0; c < 5; ++c) {
        cplx v[5] = {Cm[0][c], Cm[1][c], Cm[2][c], Cm[3][c], Cm[4][c]};
        capply(f, v);
#pragma unroll
        for (int rr = 0; rr < 5; ++rr) {
          cp[rr][c] = v[rr];
          scr(i, V_C + 2 * (5 * rr + c)) = v[rr].re;
          scr(i, V_C + 2 * (5 * rr + c) + 1) = v[rr].im;
        }
      }
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        cplx v[5] = {rhs[0][c], rhs[1][c], rhs[2][c], rhs[3][c], rhs[4][c]};
        capply(f, v);
#pragma unroll
        for (int rr = 0; rr < 5; ++rr) {
          dp[rr][c] = v[rr];
          scr(i, V_D + 2 * (NC * rr + c)) = v[rr].re;
          scr(i, V_D + 2 * (NC * rr + c) + 1) = v[rr].im;
        }
      }
    }
    // ---- back substitution, and the slots' Schur complement D - W^T X_U
    // (the held slots, without ions, an identity row)
    cplx SM[K][K], sr[K];
#pragma unroll
    for (int q = 0; q < K; ++q) {
      sr[q] = mk(0.0);
#pragma unroll
      for (int c = 0; c < K; ++c) SM[q][c] = mk(q == c && !(L.tot[q] > 0.0) ? 1.0 : 0.0);
    }
    {
      cplx xn[5][NC];
#pragma unroll
      for (int rr = 0; rr < 5; ++rr)
#pragma unroll
        for (int c = 0; c < NC; ++c) xn[rr][c] = mk(0.0);
      for (int i = NP; i >= 1; --i) {
        cplx xi[5][NC];
#pragma unroll
        for (int rr = 0; rr < 5; ++rr)
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            cplx s = mk(scr(i, V_D + 2 * (NC * rr + c)), scr(i, V_D + 2 * (NC * rr + c) + 1));
#pragma unroll
            for (int k = 0; k < 5; ++k)
              s = s - mk(scr(i, V_C + 2 * (5 * rr + k)), scr(i, V_C + 2 * (5 * rr + k) + 1)) *
                          xn[k][c];
            xi[rr][c] = s;
          }
#pragma unroll
        for (int rr = 0; rr < 5; ++rr)
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            xn[rr][c] = xi[rr][c];
            scr(i, V_D + 2 * (NC * rr + c)) = xi[rr][c].re;
            scr(i, V_D + 2 * (NC * rr + c) + 1) = xi[rr][c].im;
          }
        // each slot's constraint row: its number in its points' ion logarithms
        const Slots si = slots_at(L, i);
        const int ja = si.a >= 0 ? si.a : -1, jc = si.c >= 0 ? L.ka + si.c : -1;
        const double w3 = r5(i, R_W3), w4 = r5(i, R_W4);
#pragma unroll
        for (int q = 0; q < K; ++q) {
          const bool an = q == ja && w3 != 0.0, ca = q == jc && w4 != 0.0;
          if (!an && !ca) continue;
          const double w = an ? w3 : w4;
          const int row = an ? 3 : 4;
          sr[q] = sr[q] - w * (row == 3 ? xi[3][0] : xi[4][0]);
#pragma unroll
          for (int c = 0; c < K; ++c)
            SM[q][c] = SM[q][c] - w * (row == 3 ? xi[3][1 + c] : xi[4][1 + c]);
        }
        // a region that reaches the contact beside this point: the contact's density in the
        // number follows this point's potential, and V_int through the contact's (-dg)
        if (i == 1 || i == NP) {
          const int c = i == 1 ? 0 : NP + 1;
          const Slots sc = slots_at(L, c);
          const double dVc = i == 1 ? 0.5 * e : -0.5 * e;
#pragma unroll
          for (int sp = 0; sp < 2; ++sp) {
            const int reg = sp == 0 ? sc.a : sc.c;
            const double wv = r5(c, CT_WV + sp);
            if (reg < 0 || wv == 0.0) continue;
            const int qq = sp == 0 ? reg : L.ka + reg;
#pragma unroll
            for (int q = 0; q < K; ++q) {
              if (q != qq) continue;
              sr[q] = sr[q] - wv * xi[0][0] + mk(wv * dVc);
#pragma unroll
              for (int cc = 0; cc < K; ++cc) SM[q][cc] = SM[q][cc] - wv * xi[0][1 + cc];
            }
          }
        }
      }
    }
    csolve<K>(SM, sr);
    // dy = X_F - X_U z, written over X_F
    for (int i = 1; i <= NP; ++i)
#pragma unroll
      for (int rr = 0; rr < 5; ++rr) {
        cplx dy = mk(scr(i, V_D + 2 * (NC * rr)), scr(i, V_D + 2 * (NC * rr) + 1));
#pragma unroll
        for (int c = 0; c < K; ++c)
          dy = dy - mk(scr(i, V_D + 2 * (NC * rr + 1 + c)), scr(i, V_D + 2 * (NC * rr + 1 + c) + 1)) *
                        sr[c];
        scr(i, V_D + 2 * (NC * rr)) = dy.re;
        scr(i, V_D + 2 * (NC * rr) + 1) = dy.im;
      }
    // ---- the current's tangent: the carriers' and the displacement current as without ions,
    // then each ion region's (its base and per-dt parts)
    auto dyv = [&](int k, int c) -> cplx {
      if (k < 1 || k > NP) return mk(0.0);
      return mk(scr(k, V_D + 2 * (NC * c)), scr(k, V_D + 2 * (NC * c) + 1));
    };
    auto dV = [&](int k) -> cplx {
      if (k == 0) return mk(0.5 * e);
      if (k == NP + 1) return mk(-0.5 * e);
      return dyv(k, 0);
    };
    const double sign = -L.left();
    const double Vt = L.Vt;
    cplx dsgl[2] = {mk(0.0), mk(0.0)}, ddb_b[2] = {mk(0.0), mk(0.0)}, ddb_t[2] = {mk(0.0), mk(0.0)};
    cplx diu_b[2] = {mk(0.0), mk(0.0)}, diu_t[2] = {mk(0.0), mk(0.0)};
    cplx dS_b[2] = {mk(0.0), mk(0.0)}, dS_t[2] = {mk(0.0), mk(0.0)};
    cplx sumJ_b[2] = {mk(0.0), mk(0.0)}, sumJ_t[2] = {mk(0.0), mk(0.0)};
    cplx duc_prev_b[2] = {mk(0.0), mk(0.0)}, duc_prev_t[2] = {mk(0.0), mk(0.0)};
    cplx dJD = mk(0.0);
    // the ions, per region (slot; anion slots first): sums over the region's intervals. The
    // current of a step (dti = 1) and the steady one (dti = 0) differ where a region reaches a
    // contact: its density there `_ion_full`'s of each (R, B), and its change over the step from
    // a density of 1 before it (`_full`'s masked contact) in the integrand (values `iu_v`,
    // `dbl_v`)
    double is_[K], iH[K], aevB_f[K], aevB_l[K], aevR_f[K], aevR_l[K], iu_v[K], dbl_v[K];
    cplx dis[K], diu_i[K], ddbl_i[K], dP_i[K], dsum_i[K];
    cplx daevB_f[K], daevB_l[K], daevR_f[K], daevR_l[K];
    int first_i[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
      is_[j] = 0.0; iH[j] = 0.0; aevB_f[j] = 0.0; aevB_l[j] = 0.0; aevR_f[j] = 0.0;
      aevR_l[j] = 0.0; iu_v[j] = 0.0; dbl_v[j] = 0.0;
      dis[j] = mk(0.0); diu_i[j] = mk(0.0); ddbl_i[j] = mk(0.0); dP_i[j] = mk(0.0);
      dsum_i[j] = mk(0.0); daevB_f[j] = mk(0.0); daevB_l[j] = mk(0.0); daevR_f[j] = mk(0.0);
      daevR_l[j] = mk(0.0);
      first_i[j] = -1;
    }
    double hsum = 0.0, dx_prev = 0.0, h_prev = 0.0;
    // `currDiffInt = 1`: each interval's Scharfetter-Gummel flux for the carriers and the ions
    // (jaxdd batch.py:366-369, 471-479), from the points at both ends of the interval
    const bool cdiff = L.sc(C_CURRDIFF) > 0.0;
    cplx jd_prev[2] = {mk(0.0), mk(0.0)}, jdiB_prev[K], jdiR_prev[K], dsumdB_i[K], dsumdR_i[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
      jdiB_prev[j] = mk(0.0); jdiR_prev[j] = mk(0.0); dsumdB_i[j] = mk(0.0); dsumdR_i[j] = mk(0.0);
    }
    Pt Pa, Pb;
    if (cdiff) point(L, 0, Vint, Pa);
    for (int k = 0; k <= NP; ++k) {
      const double hk = L.st(k, S_H);
      const double dx = k < NP ? L.st(k, S_DX) : 0.0;
      const double wk = 0.5 * (dx_prev + dx);
      const double width = k == 0 ? hk : 0.5 * (h_prev + hk);
      hsum += hk;
      cplx dRi_k[2] = {mk(0.0), mk(0.0)}, dRi_k1[2] = {mk(0.0), mk(0.0)};
      bool trapped = false;
      for (int ee = k - 1; ee <= k + 1; ++ee)
        if (ee >= 0 && ee <= NP && (int)L.st(ee, S_IFK) >= 0) trapped = true;
      if (trapped) {
        const cplx ln[3] = {dyv(k - 1, 1), dyv(k, 1), dyv(k + 1, 1)};
        const cplx lp[3] = {dyv(k - 1, 2), dyv(k, 2), dyv(k + 1, 2)};
        iface_tangent(L, k, Vint, lap, a.dt, ln, lp, dRi_k[0], dRi_k[1]);
        if (k + 1 <= NP + 1) {
          const cplx ln1[3] = {dyv(k, 1), dyv(k + 1, 1), dyv(k + 2, 1)};
          const cplx lp1[3] = {dyv(k, 2), dyv(k + 1, 2), dyv(k + 2, 2)};
          iface_tangent(L, k + 1, Vint, lap, a.dt, ln1, lp1, dRi_k1[0], dRi_k1[1]);
        }
      }
      cplx dU[2] = {mk(0.0), mk(0.0)};
      if (k >= 1) {
        const double ta = rec(k, P_TA);
        cplx h, hc_unused;
        transfer(ta, lap, a.dt, h, hc_unused);
        const cplx df = ((rec(k, P_TDN) / ta) * h) * dyv(k, 1) + ((rec(k, P_TDP) / ta) * h) * dyv(k, 2);
        dU[0] = rec(k, P_TRN) * df;
        dU[1] = rec(k, P_TRP) * df;
      }
      const bool iface_k = L.st(k, S_IFK) > -1.5;
      if (cdiff) point(L, k + 1, Vint, Pb);
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const double sn = c == 0 ? -1.0 : 1.0;
        const double ev = rec(k, c == 0 ? P_EVN : P_EVP), iu = rec(k, c == 0 ? P_IUN : P_IUP);
        const double mu = L.st(k, c == 0 ? S_MUN : S_MUP);
        const cplx dev = (ev * sn / Vt) * dV(k);
        cplx duc_b = mk(0.0), duc_t = mk(0.0);
        if (k >= 1) {
          duc_b = rec(k, P_DRN) * dyv(k, 1) + rec(k, P_DRP) * dyv(k, 2) + dRi_k[c] + dU[c];
          duc_t = rec(k, c == 0 ? P_N : P_P) * dyv(k, 1 + c);
          diu_b[c] = diu_b[c] + (0.5 * dx_prev) * (duc_prev_b[c] + duc_b);
          diu_t[c] = diu_t[c] + (0.5 * dx_prev) * (duc_prev_t[c] + duc_t);
        }
        dsgl[c] = dsgl[c] + (wk / mu) * dev;
        ddb_b[c] = ddb_b[c] + (wk * iu / mu) * dev + (wk * ev / mu) * diu_b[c];
        ddb_t[c] = ddb_t[c] + (wk * ev / mu) * diu_t[c];
        const cplx dS_prev_b = dS_b[c], dS_prev_t = dS_t[c];
        if (k >= 1) {
          dS_b[c] = dS_b[c] + (sn * Q * L.L * width) * duc_b;
          dS_t[c] = dS_t[c] + (sn * Q * L.L * width) * duc_t;
        }
        const cplx thr = (sn * 0.5 * Q * L.L * hk) * (dRi_k[c] + dRi_k1[c]);
        if (cdiff) {  // as without ions
          const double d0 = c == 0 ? Pa.n : Pa.p, d1 = c == 0 ? Pb.n : Pb.p;
          const double g0 = Pa.V + (c == 0 ? Pa.offn : Pa.offp);
          const double g1 = Pb.V + (c == 0 ? Pb.offn : Pb.offp);
          double bf, bb, dbf, dbb;
          bern_pair(sn * (g1 - g0) / Vt, L.simss, bf, bb, dbf, dbb);
          const cplx dxk = (sn / Vt) * (dV(k + 1) - dV(k));
          const cplx djd = (sn * Q * mu * Vt / (L.L * hk)) *
                           (d1 * (bb * dyv(k + 1, 1 + c) - dbb * dxk) -
                            d0 * (bf * dyv(k, 1 + c) + dbf * dxk));
          sumJ_b[c] = sumJ_b[c] + hk * (iface_k ? jd_prev[c] + thr : djd);
          jd_prev[c] = djd;
        } else if (iface_k) {
          sumJ_b[c] = sumJ_b[c] + hk * (dS_prev_b + thr);
          sumJ_t[c] = sumJ_t[c] + hk * dS_prev_t;
        } else {
          sumJ_b[c] = sumJ_b[c] + hk * dS_b[c];
          sumJ_t[c] = sumJ_t[c] + hk * dS_t[c];
        }
        duc_prev_b[c] = duc_b;
        duc_prev_t[c] = duc_t;
      }
      const double epsk = W.x(k, tr::T_EPS);
      dJD = dJD + (hk * sign * epsk / (L.L * hk)) * (dV(k + 1) - dV(k));
      // the ions over interval k (points k, k+1): `_ion_currents` linearised at the state
      const Slots sa = slots_at(L, k), sb = slots_at(L, k + 1);
      // the ions' trapezoids take every interval, the last one (to the right contact) too
      const double dxi = k < NP ? dx : hk * L.L;
#pragma unroll
      for (int j = 0; j < K; ++j) {
        if (!(L.tot[j] > 0.0)) continue;
        const int sp = j < L.ka ? 0 : 1, reg = sp == 0 ? j : j - L.ka;
        const double sn = sp == 0 ? -1.0 : 1.0;
        const bool ina = (sp == 0 ? sa.a : sa.c) == reg, inb = (sp == 0 ? sb.a : sb.c) == reg;
        if (!ina && !inb) continue;
        const int tf = sp == 0 ? tr::T_MUA : tr::T_MUC;
        const double eva = r5(k, sp == 0 ? R_EVA : R_EVC), evb = r5(k + 1, sp == 0 ? R_EVA : R_EVC);
        const cplx deva = (eva * sn / Vt) * dV(k), devb = (evb * sn / Vt) * dV(k + 1);
        // each point's density and d ln(density), the step's (R) and the steady state's (B):
        // a contact's from its neighbour's, an inner point's its own
        double nBa, nRa, nBb, nRb;
        cplx dBa, dRa, dBb, dRb;
        auto end_point = [&](int pt, double& nB, double& nR, cplx& dB, cplx& dR) {
          const int nbp = pt == 0 ? 1 : NP;
          const cplx dl = dyv(nbp, 3 + sp), dv = dV(nbp) - dV(pt);
          nB = exp(r5(pt, CT_LNB + sp));
          nR = exp(r5(pt, CT_LNR + sp));
          dB = dl + ((sp == 0 ? -1.0 : 1.0) / Vt) * dv;
          dR = dl + r5(pt, CT_SR + sp) * dv;
        };
        if (k == 0) end_point(0, nBa, nRa, dBa, dRa);
        else { nBa = nRa = r5(k, sp == 0 ? R_NA : R_NC); dBa = dRa = dyv(k, 3 + sp); }
        if (k + 1 == NP + 1) end_point(NP + 1, nBb, nRb, dBb, dRb);
        else { nBb = nRb = r5(k + 1, sp == 0 ? R_NA : R_NC); dBb = dRb = dyv(k + 1, 3 + sp); }
        if (ina && first_i[j] < 0) {
          first_i[j] = k;
          aevB_f[j] = nBa * eva;
          daevB_f[j] = (nBa * eva) * dBa + nBa * deva;
          aevR_f[j] = nRa * eva;
          daevR_f[j] = (nRa * eva) * dRa + nRa * deva;
        }
        if (inb) {
          aevB_l[j] = nBb * evb;
          daevB_l[j] = (nBb * evb) * dBb + nBb * devb;
          aevR_l[j] = nRb * evb;
          daevR_l[j] = (nRb * evb) * dRb + nRb * devb;
        }
        if (cdiff) {  // the region's flux on interval k; across an interface the one before it
          double bf, bb, dbf, dbb;
          bern_pair(sn * (Pb.V - Pa.V) / Vt, L.simss, bf, bb, dbf, dbb);
          const cplx dxk = (sn / Vt) * (dV(k + 1) - dV(k));
          const double pre = sn * Q * W.x(k, tf) * Vt / (L.L * hk);
          const cplx jB = pre * ((nBb * bb) * dBb - (nBb * dbb) * dxk - (nBa * bf) * dBa -
                                 (nBa * dbf) * dxk);
          const cplx jR = pre * ((nRb * bb) * dRb - (nRb * dbb) * dxk - (nRa * bf) * dRa -
                                 (nRa * dbf) * dxk);
          if (ina && inb) {
            dsumdB_i[j] = dsumdB_i[j] + hk * (iface_k ? jdiB_prev[j] : jB);
            dsumdR_i[j] = dsumdR_i[j] + hk * (iface_k ? jdiR_prev[j] : jR);
          }
          jdiB_prev[j] = jB;
          jdiR_prev[j] = jR;
        }
        if (ina && inb) {
          const double mua = W.x(k, tf), mub = W.x(k + 1, tf);
          const double ia = 1.0 / (mua > 0.0 ? mua : 1.0), ib = 1.0 / (mub > 0.0 ? mub : 1.0);
          const cplx dUa = nRa * dRa, dUb = nRb * dRb;  // per unit of dti
          const double Uva = k == 0 ? nRa - 1.0 : 0.0, Uvb = k + 1 == NP + 1 ? nRb - 1.0 : 0.0;
          const cplx diu_b2 = diu_i[j] + (0.5 * dxi) * (dUa + dUb);
          const double iu_b2 = iu_v[j] + 0.5 * dxi * (Uva + Uvb);
          is_[j] += 0.5 * dxi * (eva * ia + evb * ib);
          dis[j] = dis[j] + (0.5 * dxi) * (ia * deva + ib * devb);
          dbl_v[j] += 0.5 * dxi * (eva * ia * iu_v[j] + evb * ib * iu_b2);
          ddbl_i[j] = ddbl_i[j] + (0.5 * dxi * eva * ia) * diu_i[j] + (0.5 * dxi * evb * ib) * diu_b2 +
                      (0.5 * dxi * ia * iu_v[j]) * deva + (0.5 * dxi * ib * iu_b2) * devb;
          diu_i[j] = diu_b2;
          iu_v[j] = iu_b2;
          const cplx dstep = k > first_i[j] ? (sn * Q * L.L * width) * dUa : mk(0.0);
          dP_i[j] = dP_i[j] + dstep;
          iH[j] += hk;
          dsum_i[j] = dsum_i[j] + hk * (iface_k ? dP_i[j] - dstep : dP_i[j]);
        }
      }
      dx_prev = dx;
      h_prev = hk;
      if (cdiff) Pa = Pb;
    }
    cplx Yb = mk(0.0), Yt = mk(0.0);
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const double sn = c == 0 ? -1.0 : 1.0;
      const double sgl = a.lsc[(size_t)(L_SN + c) * a.Bp + l], Kc = a.lsc[(size_t)(L_KN + c) * a.Bp + l];
      Pt P0, PR;
      point(L, 0, Vint, P0);
      point(L, NP + 1, Vint, PR);
      const double d0 = c == 0 ? P0.n : P0.p, dR = c == 0 ? PR.n : PR.p;
      const double e0 = exp(sn * ((c == 0 ? P0.offn : P0.offp) + P0.V) / Vt);
      const double eR = exp(sn * ((c == 0 ? PR.offn : PR.offp) + PR.V) / Vt);
      const cplx dBc = (Vt * sn) * ((dR * eR * sn / Vt) * dV(NP + 1) - (d0 * e0 * sn / Vt) * dV(0));
      const cplx dK_b = (1.0 / sgl) * (dBc - sn * ddb_b[c]) - (Kc / sgl) * dsgl[c];
      const cplx dK_t = (-sn / sgl) * ddb_t[c];
      if (!cdiff) {  // the differential current has no K
        Yb = Yb + sign * (Q * hsum) * dK_b;
        Yt = Yt + sign * (Q * hsum) * dK_t;
      }
      Yb = Yb + sign * sumJ_b[c];
      Yt = Yt + sign * sumJ_t[c];
    }
#pragma unroll
    for (int j = 0; j < K; ++j) {
      if (!(L.tot[j] > 0.0) || first_i[j] < 0) continue;
      if (cdiff) {  // the steady state's fluxes, and the step's less them per unit of dti
        Yb = Yb + sign * dsumdB_i[j];
        Yt = Yt + sign * (dsumdR_i[j] - dsumdB_i[j]);
        continue;
      }
      const double sn = j < L.ka ? -1.0 : 1.0;
      const double sgl = is_[j] > 0.0 ? is_[j] : 1.0;
      // K at dti = 0 (the steady state's) and at dti = 1, and their tangents
      const double K0 = Vt * sn * (aevB_l[j] - aevB_f[j]) / sgl;
      const double K1 = (Vt * sn * (aevR_l[j] - aevR_f[j]) - sn * dbl_v[j]) / sgl;
      const cplx dK0 = (Vt * sn / sgl) * (daevB_l[j] - daevB_f[j]) - (K0 / sgl) * dis[j];
      const cplx dK1 = (1.0 / sgl) * ((Vt * sn) * (daevR_l[j] - daevR_f[j]) - sn * ddbl_i[j]) -
                       (K1 / sgl) * dis[j];
      Yb = Yb + sign * (Q * iH[j]) * dK0;
      Yt = Yt + sign * ((Q * iH[j]) * (dK1 - dK0) + dsum_i[j]);
    }
    Yt = Yt + dJD;
    const cplx Y = (1.0 / hsum) * (Yb + lap * Yt);
    a.Y[((size_t)q * 2) * a.Bp + l] = Y.re;
    a.Y[((size_t)q * 2 + 1) * a.Bp + l] = Y.im;
  }
}

}  // namespace imp
}  // namespace dd

namespace {
long imp_threads() { return 148L * 256; }
long imp_ion_threads() { return 148L * 128; }
}

extern "C" {

int dd_admittance_workspace_bytes(const dd_batch* batch, int n_freq, size_t* bytes) {
  if (!batch || !bytes || n_freq < 1 || batch->n_lanes < 1 || batch->lane_stride % 32 != 0 ||
      batch->np_max < 3)
    return DD_ERR_ARGS;
  const size_t nodes = (size_t)batch->np_max + 2, Bp = batch->lane_stride;
  long T = (long)Bp * n_freq;
  if (T > imp_threads()) T = imp_threads();
  *bytes = (nodes * dd::imp::P_WORDS * Bp + dd::imp::L_WORDS * Bp +
            nodes * dd::imp::W_WORDS * (size_t)T) * sizeof(double);
  return DD_OK;
}

int dd_admittance(const dd_batch* batch, const double* state, const double* eps,
                  const double* vint, const double* laps, int n_freq, int bernoulli, double dt,
                  double* Y, void* workspace, size_t workspace_bytes, void* stream) {
  if (!batch || !batch->stat || !batch->scal || !batch->iface || !state || !eps || !vint ||
      !laps || n_freq < 1 || !Y || !workspace)
    return DD_ERR_ARGS;
  if (batch->n_lanes < 1 || batch->lane_stride < batch->n_lanes || batch->lane_stride % 32 != 0 ||
      batch->np_max < 3 || batch->k_anion != 1 || batch->k_cation != 1)
    return DD_ERR_ARGS;
  if (bernoulli != DD_BERNOULLI_EXACT && bernoulli != DD_BERNOULLI_SIMSS) return DD_ERR_ARGS;
  size_t need;
  dd_admittance_workspace_bytes(batch, n_freq, &need);
  if (workspace_bytes < need) return DD_ERR_WORKSPACE;
  const size_t nodes = (size_t)batch->np_max + 2, Bp = batch->lane_stride;
  dd::imp::Args a{};
  a.B = batch->n_lanes; a.Bp = batch->lane_stride; a.npmax = batch->np_max; a.ka = batch->k_anion;
  a.simss = bernoulli == DD_BERNOULLI_SIMSS; a.nf = n_freq;
  if (dt < 0.0) return DD_ERR_ARGS;
  a.dt = dt;
  a.S = batch->stat; a.C = batch->scal; a.IFt = batch->iface;
  a.state = state; a.eps = eps; a.vint = vint; a.laps = laps; a.Y = Y;
  double* ws = static_cast<double*>(workspace);
  a.rec = ws;
  a.lsc = ws + nodes * dd::imp::P_WORDS * Bp;
  a.scr = a.lsc + dd::imp::L_WORDS * Bp;
  long T = (long)Bp * n_freq;
  if (T > imp_threads()) T = imp_threads();
  a.T = T;
  int st = dd::device_status();
  if (st != DD_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  st = dd::launch(dd::imp::prepare_kernel, dim3((unsigned)((Bp + 63) / 64)), dim3(64), 0, s, a);
  if (st == DD_OK)
    st = dd::launch(dd::imp::admittance_kernel, dim3((unsigned)((T + 63) / 64)), dim3(64), 0, s, a);
  return st;
}

int dd_admittance_ions_workspace_bytes(const dd_batch* batch, int n_freq, size_t* bytes) {
  if (!batch || !bytes || n_freq < 1 || batch->n_lanes < 1 || batch->lane_stride % 32 != 0 ||
      batch->np_max < 3)
    return DD_ERR_ARGS;
  const size_t nodes = (size_t)batch->np_max + 2, Bp = batch->lane_stride;
  long T = (long)Bp * n_freq;
  if (T > imp_ion_threads()) T = imp_ion_threads();
  const int K = batch->k_anion + batch->k_cation;
  if (batch->k_anion < 1 || batch->k_cation < 1 || K > dd::DD_MAXK) return DD_ERR_ARGS;
  *bytes = (nodes * dd::imp::P_WORDS * Bp + dd::imp::L_WORDS * Bp +
            nodes * dd::imp::R5_WORDS * Bp + nodes * dd::imp::vwords(K) * (size_t)T) *
           sizeof(double);
  return DD_OK;
}

int dd_admittance_ions(const dd_batch* batch, const double* state, const double* state_logs,
                       const double* tstat, const double* vint, const double* laps, int n_freq,
                       int bernoulli, double dt, double* Y, void* workspace,
                       size_t workspace_bytes, void* stream) {
  if (!batch || !batch->stat || !batch->scal || !batch->iface || !state || !state_logs ||
      !tstat || !vint || !laps || n_freq < 1 || !Y || !workspace)
    return DD_ERR_ARGS;
  if (batch->n_lanes < 1 || batch->lane_stride < batch->n_lanes || batch->lane_stride % 32 != 0 ||
      batch->np_max < 3)
    return DD_ERR_ARGS;
  if (bernoulli != DD_BERNOULLI_EXACT && bernoulli != DD_BERNOULLI_SIMSS) return DD_ERR_ARGS;
  size_t need;  // (the slots: k_anion, k_cation >= 1, at most DD_MAXK in all)
  if (dd_admittance_ions_workspace_bytes(batch, n_freq, &need) != DD_OK) return DD_ERR_ARGS;
  if (workspace_bytes < need) return DD_ERR_WORKSPACE;
  const size_t nodes = (size_t)batch->np_max + 2, Bp = batch->lane_stride;
  dd::imp::Args a{};
  a.B = batch->n_lanes; a.Bp = batch->lane_stride; a.npmax = batch->np_max; a.ka = batch->k_anion;
  a.K = batch->k_anion + batch->k_cation;
  a.simss = bernoulli == DD_BERNOULLI_SIMSS; a.nf = n_freq;
  if (dt < 0.0) return DD_ERR_ARGS;
  a.dt = dt;
  a.S = batch->stat; a.C = batch->scal; a.IFt = batch->iface;
  a.state = state; a.eps = nullptr; a.vint = vint; a.laps = laps; a.Y = Y;
  double* ws = static_cast<double*>(workspace);
  a.rec = ws;
  a.lsc = ws + nodes * dd::imp::P_WORDS * Bp;
  dd::imp::IonArgs b{};
  b.X = tstat;
  b.state_logs = state_logs;
  b.rec5 = a.lsc + dd::imp::L_WORDS * Bp;
  b.scr5 = b.rec5 + nodes * dd::imp::R5_WORDS * Bp;
  a.scr = nullptr;
  long T = (long)Bp * n_freq;
  if (T > imp_ion_threads()) T = imp_ion_threads();
  a.T = T;
  int st = dd::device_status();
  if (st != DD_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  st = dd::launch(dd::imp::prepare_kernel, dim3((unsigned)((Bp + 63) / 64)), dim3(64), 0, s, a);
  if (st != DD_OK) return st;
  const dim3 gp((unsigned)((Bp + 31) / 32)), ga((unsigned)((T + 63) / 64));
  switch (a.K) {  // the slots: one region of each species, or several
    case 2:
      st = dd::launch(dd::imp::prepare_ions_kernel<2>, gp, dim3(32), 0, s, a, b);
      if (st == DD_OK) st = dd::launch(dd::imp::admittance_ions_kernel<2>, ga, dim3(64), 0, s, a, b);
      break;
    case 3:
      st = dd::launch(dd::imp::prepare_ions_kernel<3>, gp, dim3(32), 0, s, a, b);
      if (st == DD_OK) st = dd::launch(dd::imp::admittance_ions_kernel<3>, ga, dim3(64), 0, s, a, b);
      break;
    default:
      st = dd::launch(dd::imp::prepare_ions_kernel<4>, gp, dim3(32), 0, s, a, b);
      if (st == DD_OK) st = dd::launch(dd::imp::admittance_ions_kernel<4>, ga, dim3(64), 0, s, a, b);
  }
  return st;
}

}  // extern "C"
