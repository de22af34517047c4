// TEST INFRASTRUCTURE ONLY — FP64 C++ restatement of the oracle's `solve_batch` (oracle/dd.py),
// itself a restatement of jaxdd's batched J-V solve (src/jaxdd/batch.py:1136-1208 and the solver
// functions it calls). One device at a time, single-threaded, scalar code: what jaxdd's CPU path
// computes for one device, in the form a compiled CPU implementation of it takes. It is the CPU
// baseline the benchmark times (one process per host core) and a second checker of the CUDA
// path; nothing in the product links it. Pinned to oracle/dd.py by tests/test_oracle_cpu.py
// (J within 1e-10 of the current scale, converged flags equal).
//
// Each function names the oracle function and the reference lines it follows. The 3x3 block
// solves use LU with partial pivoting, as the oracle's np.linalg.solve (LAPACK gesv) does.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

extern "C" {

// One device's tree (oracle/dd.py `_one`, the scope of the CUDA path), pointers into the
// caller's arrays. Interior arrays have NP entries (points 1..NP), point arrays NP + 2,
// interval arrays NP + 1.
struct ddc_device {
  int32_t NP, ka, kc, pad;
  // interior stencils and row data (`_stencils`, solver.py:210-278)
  const double *fac_l, *fac_m, *fac_u, *fac, *sP, *sC, *dop, *a_mask, *c_mask, *a_fix, *c_fix;
  // points
  const double *x, *h, *N_c, *ni, *E_c, *offset_n, *offset_p, *mu_n, *mu_p, *G;
  const double *kd, *ni2, *Nt, *Cn, *Cp, *nt0, *pt0;
  // interface traps per interval, [10][NP + 1] in oracle/dd.py's _TI_KEYS order
  const double* ti;
  const uint8_t* iface;  // [NP + 1] the interval is a layer interface
  const double* hL;      // [NP + 1] h L of each interval
  const double *a_slots, *c_slots;    // [ka][NP + 2], [kc][NP + 2]
  const double *a_totals, *c_totals;  // [ka], [kc]
  double Vt, g_frac, L, V0, VL, W_L, W_R, ln_n_left, ln_n_right, ln_p_left, ln_p_right;
  double J_scale, left_elec, G_shunt, pre_cond, V_pre, fix_ions, curr_diff, n_floor;
};

int ddc_solve_batch(const ddc_device* dev, const double* voltages, int nv, double tol,
                    int max_iter, int first_max_iter, int simss, double* J, uint8_t* converged,
                    int32_t* iterations);
}

namespace {

constexpr double Q = 1.6022e-19;
constexpr double ROUND_OFF_FLOOR = 1e-6;
constexpr int STALL_STEPS = 3;
constexpr double CAPS[3] = {10.0, 5.0, 5.0};
constexpr double ION_LOG_CAP = 5.0;
constexpr double FLOOR_DROP_CAP = 50.0;
constexpr double CURRENT_TOL = 1e-5;
constexpr double CURRENT_STEP_CAP = 1e-3;
constexpr double QUADRATIC_TOL = 1e-5;
constexpr double QUADRATIC_RATIO = 1e-2;
constexpr double STAGES[4] = {1.0 / 64, 1.0 / 16, 1.0 / 4, 1.0};
constexpr double SERIES_BELOW = 1e-2;
constexpr int TI_NT = 0, TI_CN = 1, TI_CP = 2, TI_NT0LO = 3, TI_PT0LO = 4, TI_NT0HI = 5,
              TI_PT0HI = 6, TI_IW = 7, TI_CHARGE = 8, TI_CWE = 9;

using Vec = std::vector<double>;

// np.maximum / np.max: a NaN anywhere stays
inline double nmax(double a, double b) { return (std::isnan(a) || std::isnan(b)) ? NAN : (a > b ? a : b); }
inline double clip(double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); }

// `bern_exact` (solver.py:95-105) and `bern_simss` (solver.py:108-121) with their derivatives
void bern(double x, bool simss, double& b, double& db) {
  const double ax = std::fabs(x);
  if (!simss) {
    if (ax < SERIES_BELOW) {
      b = 1.0 - x / 2.0 + x * x / 12.0 - (x * x * x * x) / 720.0;
      db = -0.5 + x / 6.0 - (x * x * x) / 180.0;
      return;
    }
  } else {
    if (ax < 0.05) { b = 1.0 - 0.5 * x; db = -0.5; return; }
    if (ax < 0.45) { b = 1.0 - x * (0.5 - x / 12.0); db = -0.5 + x / 6.0; return; }
    if (ax < 1.5) {
      b = 1.0 + x * (-0.5 + x * (1.0 / 12.0 - x * x / 720.0));
      db = -0.5 + x / 6.0 - (x * x * x) / 180.0;
      return;
    }
  }
  const double e = std::expm1(x);
  b = x / e;
  db = 1.0 / e - x * (e + 1.0) / (e * e);
}

// A device's mutable view: the scaled or frozen ions (`_scaled`, `freeze`) change these.
struct Model {
  const ddc_device* d;
  int NP, K, ka;
  bool simss;
  Vec a_fix, c_fix, a_mask, c_mask;  // interior
  Vec masks;                         // [K][NP + 2], anion slots first
  Vec totals, sign;                  // [K]
  bool any_traps;

  explicit Model(const ddc_device* dv, bool sim) : d(dv), NP(dv->NP), K(dv->ka + dv->kc), ka(dv->ka), simss(sim) {
    a_fix.assign(dv->a_fix, dv->a_fix + NP);
    c_fix.assign(dv->c_fix, dv->c_fix + NP);
    a_mask.assign(dv->a_mask, dv->a_mask + NP);
    c_mask.assign(dv->c_mask, dv->c_mask + NP);
    masks.resize((size_t)K * (NP + 2));
    totals.resize(K);
    sign.resize(K);
    for (int k = 0; k < K; ++k) {
      const bool an = k < ka;
      const double* src = an ? dv->a_slots + (size_t)k * (NP + 2) : dv->c_slots + (size_t)(k - ka) * (NP + 2);
      std::memcpy(&masks[(size_t)k * (NP + 2)], src, sizeof(double) * (NP + 2));
      totals[k] = an ? dv->a_totals[k] : dv->c_totals[k - ka];
      sign[k] = an ? 1.0 : -1.0;
    }
    any_traps = false;
    for (int e = 0; e <= NP; ++e) any_traps = any_traps || dv->ti[(size_t)TI_NT * (NP + 1) + e] > 0.0;
  }
  double ti(int f, int e) const { return d->ti[(size_t)f * (NP + 1) + e]; }
  double mask(int k, int i) const { return masks[(size_t)k * (NP + 2) + i]; }
  bool mobile() const {
    for (int k = 0; k < K; ++k)
      if (totals[k] > 0.0) return true;
    return false;
  }
};

// `_recombination` (solver.py:734-745): R and n dR/dn, p dR/dp at point i
void recombination(const ddc_device* d, int i, double n, double p, double& R, double& dRn, double& dRp) {
  const double Nt = d->Nt[i], Cn = d->Cn[i], Cp = d->Cp[i], nt0 = d->nt0[i], pt0 = d->pt0[i];
  const bool traps = Nt > 0.0;
  const double num = Nt * Cn * Cp * (n * p - nt0 * pt0);
  const double den = traps ? Cn * (n + nt0) + Cp * (p + pt0) : 1.0;
  const double srh = traps ? num / den : 0.0;
  R = d->kd[i] * (n * p - d->ni2[i]) + srh;
  const double dsn = traps ? (Nt * Cn * Cp * p - srh * Cn) / den : 0.0;
  const double dsp = traps ? (Nt * Cn * Cp * n - srh * Cp) / den : 0.0;
  dRn = n * (d->kd[i] * p + dsn);
  dRp = p * (d->kd[i] * n + dsp);
}

// `_iface_edges` (solver.py:814-850): interval e's values (Rn_L, Rn_R, Rp_L, Rp_R, Q) and their
// derivatives in ln nL, ln nR, ln pL, ln pR
void iface_edge(const Model& m, int e, double nL, double nR, double pL, double pR, double (&val)[5],
                double (&der)[4][5]) {
  const double Nt = m.ti(TI_NT, e), Cn = m.ti(TI_CN, e), Cp = m.ti(TI_CP, e), iw = m.ti(TI_IW, e);
  const double nlo = m.ti(TI_NT0LO, e), nhi = m.ti(TI_NT0HI, e);
  const double plo = m.ti(TI_PT0LO, e), phi = m.ti(TI_PT0HI, e);
  const double an = Cn * Nt, bp = Cp * Nt;
  const bool traps = Nt > 0.0;
  const double a = an * (nL + nR), b = bp * (pL + pR), c = an * (nlo + nhi), dd = bp * (plo + phi);
  const double S = traps ? a + b + c + dd : 1.0;
  const double inv = traps ? 1.0 / S : 0.0;
  const double full = (a + dd) * inv, empty = (b + c) * inv;
  const double half_q = m.ti(TI_CHARGE, e) * 0.5 * Nt * iw;
  val[0] = iw * an * (nL * empty - nlo * full);
  val[1] = iw * an * (nR * empty - nhi * full);
  val[2] = iw * bp * (pL * full - plo * empty);
  val[3] = iw * bp * (pR * full - phi * empty);
  val[4] = half_q * (m.ti(TI_CWE, e) - full);
  for (int w = 0; w < 4; ++w) {
    double dfull, dempty;
    if (w < 2) {
      const double da = an * (w == 0 ? nL : nR);
      dfull = da * empty * inv; dempty = -da * empty * inv;
    } else {
      const double db = bp * (w == 2 ? pL : pR);
      dfull = -db * full * inv; dempty = db * full * inv;
    }
    const double own[4] = {w == 0 ? 1.0 : 0.0, w == 1 ? 1.0 : 0.0, w == 2 ? 1.0 : 0.0, w == 3 ? 1.0 : 0.0};
    der[w][0] = iw * an * (own[0] * nL * empty + nL * dempty - nlo * dfull);
    der[w][1] = iw * an * (own[1] * nR * empty + nR * dempty - nhi * dfull);
    der[w][2] = iw * bp * (own[2] * pL * full + pL * dfull - plo * dempty);
    der[w][3] = iw * bp * (own[3] * pR * full + pR * dfull - phi * dempty);
    der[w][4] = -half_q * dfull;
  }
}

// The system of one Newton step (`system`, batch.py:518-549 via oracle/dd.py): residual F, blocks
// A, B, C, slot columns U (NP x 3 x K), the constraints g, border W (K x NP), D (K x K diagonal).
struct System {
  int NP, K;
  Vec F, A, B, C, U, g, W, D;
  void size(int np, int k) {
    NP = np; K = k;
    F.assign((size_t)NP * 3, 0.0); A.assign((size_t)NP * 9, 0.0); B.assign((size_t)NP * 9, 0.0);
    C.assign((size_t)NP * 9, 0.0); U.assign((size_t)NP * 3 * K, 0.0); g.assign(K, 0.0);
    W.assign((size_t)K * NP, 0.0); D.assign((size_t)K * K, 0.0);
  }
};

// `point_logs` (solver.py:1201-1204): each interior point's anion and cation normalisation
void point_logs(const Model& m, const double* logs, Vec& la, Vec& lc) {
  la.assign(m.NP, 0.0); lc.assign(m.NP, 0.0);
  for (int j = 0; j < m.NP; ++j) {
    double a = 0.0, c = 0.0;
    for (int k = 0; k < m.ka; ++k) a += logs[k] * m.mask(k, j + 1);
    for (int k = m.ka; k < m.K; ++k) c += logs[k] * m.mask(k, j + 1);
    la[j] = a; lc[j] = c;
  }
}

// `_assemble` (solver.py:1021-1187 via oracle/dd.py `assemble`) and the ion constraints
// (`ion_constraints`, solver.py:1255-1265), full = (NP + 2) x 3
void assemble(const Model& m, const Vec& full, const double* logs, System& s) {
  const ddc_device* d = m.d;
  const int NP = m.NP;
  const double Vt = d->Vt;
  Vec V(NP + 2), n(NP + 2), p(NP + 2);
  for (int i = 0; i < NP + 2; ++i) { V[i] = full[3 * i]; n[i] = std::exp(full[3 * i + 1]); p[i] = std::exp(full[3 * i + 2]); }
  // interval fluxes and their derivatives
  Vec Fn(NP + 1), Fp(NP + 1), dFn0(3 * (NP + 1)), dFn1(3 * (NP + 1)), dFp0(3 * (NP + 1)), dFp1(3 * (NP + 1));
  for (int e = 0; e <= NP; ++e) {
    const double cn = Vt * d->mu_n[e], cp = Vt * d->mu_p[e];
    const double xn = ((V[e + 1] + d->offset_n[e + 1]) - (V[e] + d->offset_n[e])) / Vt;
    const double xp = ((V[e + 1] + d->offset_p[e + 1]) - (V[e] + d->offset_p[e])) / Vt;
    double Bnf, dBnf, Bnb, dBnb, Bpf, dBpf, Bpb, dBpb;
    bern(xn, m.simss, Bnf, dBnf);
    bern(-xn, m.simss, Bnb, dBnb);
    bern(xp, m.simss, Bpf, dBpf);
    bern(-xp, m.simss, Bpb, dBpb);
    const double n0 = n[e], n1 = n[e + 1], p0 = p[e], p1 = p[e + 1];
    Fn[e] = cn * (Bnf * n1 - Bnb * n0);
    const double gn = cn * (dBnf * n1 + dBnb * n0) / Vt;
    dFn0[3 * e] = -gn; dFn0[3 * e + 1] = -cn * Bnb * n0; dFn0[3 * e + 2] = 0.0;
    dFn1[3 * e] = gn; dFn1[3 * e + 1] = cn * Bnf * n1; dFn1[3 * e + 2] = 0.0;
    Fp[e] = cp * (Bpf * p0 - Bpb * p1);
    const double gp = cp * (dBpf * p0 + dBpb * p1) / Vt;
    dFp0[3 * e] = -gp; dFp0[3 * e + 1] = 0.0; dFp0[3 * e + 2] = cp * Bpf * p0;
    dFp1[3 * e] = gp; dFp1[3 * e + 1] = 0.0; dFp1[3 * e + 2] = -cp * Bpb * p1;
  }
  Vec la, lc;
  point_logs(m, logs, la, lc);
  // interface traps per interval
  Vec tval, tder;
  if (m.any_traps) {
    tval.resize((size_t)5 * (NP + 1));
    tder.resize((size_t)20 * (NP + 1));
    for (int e = 0; e <= NP; ++e) {
      double v[5], dv[4][5];
      iface_edge(m, e, n[e], n[e + 1], p[e], p[e + 1], v, dv);
      for (int q = 0; q < 5; ++q) tval[(size_t)q * (NP + 1) + e] = v[q];
      for (int w = 0; w < 4; ++w)
        for (int q = 0; q < 5; ++q) tder[((size_t)w * 5 + q) * (NP + 1) + e] = dv[w][q];
    }
  }
  auto TV = [&](int q, int e) { return tval[(size_t)q * (NP + 1) + e]; };
  auto TD = [&](int w, int q, int e) { return tder[((size_t)w * 5 + q) * (NP + 1) + e]; };
  const int lo[3] = {4, 0, 2}, hi[3] = {4, 1, 3};
  for (int j = 0; j < NP; ++j) {
    const int i = j + 1;
    const double hm = d->h[i - 1], hp = d->h[i], fac = d->fac[j];
    double R, dRn, dRp;
    recombination(d, i, n[i], p[i], R, dRn, dRp);
    const double gen = d->G[i] * d->g_frac;
    const double dnet[3] = {0.0, -dRn, -dRp};
    double elec = hm * Fn[i] - hp * Fn[i - 1] + fac * (gen - R);
    double hole = hp * Fp[i - 1] - hm * Fp[i] + fac * (gen - R);
    const double anion = m.a_mask[j] * std::exp(la[j] + V[i] / Vt);
    const double cation = m.c_mask[j] * std::exp(lc[j] - V[i] / Vt);
    double poisson = d->fac_l[j] * V[i - 1] + d->fac_m[j] * V[i] + d->fac_u[j] * V[i + 1] -
                     Q * (n[i] - p[i] + d->dop[j] + m.a_fix[j] + anion - m.c_fix[j] - cation);
    const double sP = d->sP[j], sC = d->sC[j];
    double* A = &s.A[(size_t)j * 9];
    double* B = &s.B[(size_t)j * 9];
    double* C = &s.C[(size_t)j * 9];
    const double PA[3] = {d->fac_l[j], 0.0, 0.0}, PC[3] = {d->fac_u[j], 0.0, 0.0};
    const double PB[3] = {d->fac_m[j] - Q * (anion + cation) / Vt, -Q * n[i], Q * p[i]};
    for (int c = 0; c < 3; ++c) {
      A[c] = PA[c] * sP;
      A[3 + c] = -hp * dFn0[3 * (i - 1) + c] * sC;
      A[6 + c] = hp * dFp0[3 * (i - 1) + c] * sC;
      B[c] = PB[c] * sP;
      B[3 + c] = (-hp * dFn1[3 * (i - 1) + c] + hm * dFn0[3 * i + c] + fac * dnet[c]) * sC;
      B[6 + c] = (hp * dFp1[3 * (i - 1) + c] - hm * dFp0[3 * i + c] + fac * dnet[c]) * sC;
      C[c] = PC[c] * sP;
      C[3 + c] = hm * dFn1[3 * i + c] * sC;
      C[6 + c] = -hm * dFp1[3 * i + c] * sC;
    }
    if (m.any_traps) {
      const double scale[3] = {Q * sP, -fac * sC, -fac * sC};
      double X[3];
      for (int r = 0; r < 3; ++r) X[r] = TV(hi[r], j) + TV(lo[r], j + 1);
      poisson = poisson + Q * X[0];
      elec = elec - fac * X[1];
      hole = hole - fac * X[2];
      for (int r = 0; r < 3; ++r) {
        // own: d/d(ln nR) of the left interval + d/d(ln nL) of the right one; up: the right
        // interval in its right end; down: the left interval in its left end
        const double own_n = TD(1, hi[r], j) + TD(0, lo[r], j + 1);
        const double own_p = TD(3, hi[r], j) + TD(2, lo[r], j + 1);
        const double up_n = TD(1, lo[r], j + 1), up_p = TD(3, lo[r], j + 1);
        const double dn_n = TD(0, hi[r], j), dn_p = TD(2, hi[r], j);
        A[3 * r + 1] += dn_n * scale[r]; A[3 * r + 2] += dn_p * scale[r];
        B[3 * r + 1] += own_n * scale[r]; B[3 * r + 2] += own_p * scale[r];
        C[3 * r + 1] += up_n * scale[r]; C[3 * r + 2] += up_p * scale[r];
      }
    }
    s.F[3 * j] = poisson * sP;
    s.F[3 * j + 1] = elec * sC;
    s.F[3 * j + 2] = hole * sC;
    // slot columns (`slot_columns`, solver.py:1207-1212): the Poisson row only
    for (int k = 0; k < m.K; ++k) {
      const double u = k < m.ka ? (-Q * anion) * sP : (Q * cation) * sP;
      s.U[((size_t)j * 3 + 0) * m.K + k] = u * m.mask(k, i);
      s.U[((size_t)j * 3 + 1) * m.K + k] = 0.0;
      s.U[((size_t)j * 3 + 2) * m.K + k] = 0.0;
    }
  }
  // the ions' constraints, their border and D (`ion_constraints`, `_held`)
  for (int k = 0; k < m.K; ++k) {
    Vec dens(NP + 2);
    for (int i = 0; i < NP + 2; ++i) dens[i] = m.mask(k, i) * std::exp(logs[k] + m.sign[k] * V[i] / Vt);
    double number = 0.0;
    for (int e = 0; e <= NP; ++e) {
      const double pair = m.mask(k, e + 1) * m.mask(k, e);
      number += 0.5 * (dens[e + 1] + dens[e]) * pair * d->hL[e];
    }
    const bool has = m.totals[k] > 0.0;
    const double tot = has ? m.totals[k] : 1.0;
    s.g[k] = has ? number / tot - 1.0 : 0.0;
    for (int j = 0; j < NP; ++j) {
      const double pl = m.mask(k, j + 1) * m.mask(k, j) * d->hL[j];
      const double pr = m.mask(k, j + 2) * m.mask(k, j + 1) * d->hL[j + 1];
      const double wpt = 0.5 * (pl + pr);
      s.W[(size_t)k * NP + j] = has ? wpt * dens[j + 1] * m.sign[k] / Vt / tot : 0.0;
    }
    for (int l = 0; l < m.K; ++l) s.D[(size_t)k * m.K + l] = 0.0;
    s.D[(size_t)k * m.K + k] = (has ? number / tot : 0.0) + (has ? 0.0 : 1.0);
  }
}

// M x = R for a small dense M (n x n) and R (n x c), by LU with partial pivoting (LAPACK gesv's
// algorithm: the first largest pivot). M and R are overwritten; R holds x.
void lu_solve(double* M, double* R, int n, int c) {
  for (int col = 0; col < n; ++col) {
    int piv = col;
    double best = std::fabs(M[col * n + col]);
    for (int r = col + 1; r < n; ++r)
      if (std::fabs(M[r * n + col]) > best) { best = std::fabs(M[r * n + col]); piv = r; }
    if (piv != col) {
      for (int q = 0; q < n; ++q) std::swap(M[col * n + q], M[piv * n + q]);
      for (int q = 0; q < c; ++q) std::swap(R[col * c + q], R[piv * c + q]);
    }
    const double inv = 1.0 / M[col * n + col];
    for (int r = col + 1; r < n; ++r) {
      const double f = M[r * n + col] * inv;
      M[r * n + col] = f;
      for (int q = col + 1; q < n; ++q) M[r * n + q] -= f * M[col * n + q];
      for (int q = 0; q < c; ++q) R[r * c + q] -= f * R[col * c + q];
    }
  }
  for (int r = n - 1; r >= 0; --r)
    for (int q = 0; q < c; ++q) {
      double v = R[r * c + q];
      for (int k = r + 1; k < n; ++k) v -= M[r * n + k] * R[k * c + q];
      R[r * c + q] = v / M[r * n + r];
    }
}

// `block_thomas` (solver.py:1534-1560): d is NP x 3 x mc, overwritten by the solution
void block_thomas(const System& s, Vec& dmat, int mc) {
  const int NP = s.NP;
  Vec cp((size_t)NP * 9), dp((size_t)NP * 3 * mc);
  double c_prev[9] = {0}, M[9], R[3 * (3 + 8)];
  std::vector<double> d_prev((size_t)3 * mc, 0.0);
  const int w = 3 + mc;
  for (int i = 0; i < NP; ++i) {
    const double* A = &s.A[(size_t)i * 9];
    const double* B = &s.B[(size_t)i * 9];
    const double* C = &s.C[(size_t)i * 9];
    for (int r = 0; r < 3; ++r)
      for (int q = 0; q < 3; ++q)
        M[3 * r + q] = B[3 * r + q] - (A[3 * r] * c_prev[q] + A[3 * r + 1] * c_prev[3 + q] + A[3 * r + 2] * c_prev[6 + q]);
    for (int r = 0; r < 3; ++r) {
      for (int q = 0; q < 3; ++q) R[r * w + q] = C[3 * r + q];
      for (int q = 0; q < mc; ++q)
        R[r * w + 3 + q] = dmat[((size_t)i * 3 + r) * mc + q] -
                           (A[3 * r] * d_prev[q] + A[3 * r + 1] * d_prev[mc + q] + A[3 * r + 2] * d_prev[2 * mc + q]);
    }
    lu_solve(M, R, 3, w);
    for (int r = 0; r < 3; ++r) {
      for (int q = 0; q < 3; ++q) c_prev[3 * r + q] = R[r * w + q];
      for (int q = 0; q < mc; ++q) d_prev[(size_t)r * mc + q] = R[r * w + 3 + q];
    }
    std::memcpy(&cp[(size_t)i * 9], c_prev, sizeof(c_prev));
    std::memcpy(&dp[(size_t)i * 3 * mc], d_prev.data(), sizeof(double) * 3 * mc);
  }
  std::vector<double> nxt((size_t)3 * mc, 0.0), t((size_t)3 * mc);
  for (int i = NP - 1; i >= 0; --i) {
    const double* c = &cp[(size_t)i * 9];
    for (int r = 0; r < 3; ++r)
      for (int q = 0; q < mc; ++q)
        t[(size_t)r * mc + q] = dp[((size_t)i * 3 + r) * mc + q] -
                                (c[3 * r] * nxt[q] + c[3 * r + 1] * nxt[mc + q] + c[3 * r + 2] * nxt[2 * mc + q]);
    nxt = t;
    for (size_t q = 0; q < (size_t)3 * mc; ++q) dmat[(size_t)i * 3 * mc + q] = nxt[q];
  }
}

// The mixed-precision experiment (`ddc_solve_batch_mixed`): the block sweep in FP32 — the
// inexact Newton of an FP32 Jacobian solve — after each node's unknowns and rows are scaled by
// the largest entries of its diagonal block (with rows alone the FP32 elimination overflows where
// a depleted layer's continuity rows are 1e-20 of the Poisson row). The residual, the step's
// damping and size, the current and every stop stay FP64.
void block_thomas32(const System& s, Vec& dmat, int mc) {
  // per-node column scales (node j's unknowns in units of cs[j]) and row scales, both from the
  // diagonal blocks B, then the factorisation, carries and substitutions in float
  const int NP = s.NP;
  std::vector<double> cs((size_t)NP * 3), rs((size_t)NP * 3);
  for (int i = 0; i < NP; ++i)
    for (int q = 0; q < 3; ++q) {
      double mx = 0;
      for (int r = 0; r < 3; ++r) mx = std::fmax(mx, std::fabs(s.B[(size_t)i * 9 + 3 * r + q]));
      cs[(size_t)i * 3 + q] = mx > 0 ? 1.0 / mx : 1.0;
    }
  for (int i = 0; i < NP; ++i)
    for (int r = 0; r < 3; ++r) {
      double mx = 0;
      for (int q = 0; q < 3; ++q) mx = std::fmax(mx, std::fabs(s.B[(size_t)i * 9 + 3 * r + q] * cs[(size_t)i * 3 + q]));
      rs[(size_t)i * 3 + r] = mx > 0 ? 1.0 / mx : 1.0;
    }
  std::vector<float> cp((size_t)NP * 9), dp((size_t)NP * 3 * mc);
  float c_prev[9] = {0}, M[9];
  std::vector<float> R((size_t)3 * (3 + mc)), d_prev((size_t)3 * mc, 0.f);
  const int w = 3 + mc;
  for (int i = 0; i < NP; ++i) {
    float A[9], B[9], C[9], rr[3][8];
    for (int r = 0; r < 3; ++r) {
      const double sc = rs[(size_t)i * 3 + r];
      for (int q = 0; q < 3; ++q) {
        A[3 * r + q] = i > 0 ? (float)(s.A[(size_t)i * 9 + 3 * r + q] * sc * cs[(size_t)(i - 1) * 3 + q]) : 0.f;
        B[3 * r + q] = (float)(s.B[(size_t)i * 9 + 3 * r + q] * sc * cs[(size_t)i * 3 + q]);
        C[3 * r + q] = i + 1 < NP ? (float)(s.C[(size_t)i * 9 + 3 * r + q] * sc * cs[(size_t)(i + 1) * 3 + q]) : 0.f;
      }
      for (int q = 0; q < mc; ++q) rr[r][q] = (float)(dmat[((size_t)i * 3 + r) * mc + q] * sc);
    }
    for (int r = 0; r < 3; ++r)
      for (int q = 0; q < 3; ++q)
        M[3 * r + q] = B[3 * r + q] - (A[3 * r] * c_prev[q] + A[3 * r + 1] * c_prev[3 + q] + A[3 * r + 2] * c_prev[6 + q]);
    for (int r = 0; r < 3; ++r) {
      for (int q = 0; q < 3; ++q) R[r * w + q] = C[3 * r + q];
      for (int q = 0; q < mc; ++q)
        R[r * w + 3 + q] = rr[r][q] - (A[3 * r] * d_prev[q] + A[3 * r + 1] * d_prev[mc + q] + A[3 * r + 2] * d_prev[2 * mc + q]);
    }
    for (int col = 0; col < 3; ++col) {
      int piv = col; float best = std::fabs(M[col * 3 + col]);
      for (int r = col + 1; r < 3; ++r) if (std::fabs(M[r * 3 + col]) > best) { best = std::fabs(M[r * 3 + col]); piv = r; }
      if (piv != col) { for (int q = 0; q < 3; ++q) std::swap(M[col * 3 + q], M[piv * 3 + q]); for (int q = 0; q < w; ++q) std::swap(R[col * w + q], R[piv * w + q]); }
      const float inv = 1.f / M[col * 3 + col];
      for (int r = col + 1; r < 3; ++r) { const float f = M[r * 3 + col] * inv; for (int q = col + 1; q < 3; ++q) M[r * 3 + q] -= f * M[col * 3 + q]; for (int q = 0; q < w; ++q) R[r * w + q] -= f * R[col * w + q]; }
    }
    for (int r = 2; r >= 0; --r) for (int q = 0; q < w; ++q) { float v = R[r * w + q]; for (int k = r + 1; k < 3; ++k) v -= M[r * 3 + k] * R[k * w + q]; R[r * w + q] = v / M[r * 3 + r]; }
    for (int r = 0; r < 3; ++r) {
      for (int q = 0; q < 3; ++q) c_prev[3 * r + q] = R[r * w + q];
      for (int q = 0; q < mc; ++q) d_prev[(size_t)r * mc + q] = R[r * w + 3 + q];
    }
    std::memcpy(&cp[(size_t)i * 9], c_prev, sizeof(c_prev));
    std::memcpy(&dp[(size_t)i * 3 * mc], d_prev.data(), sizeof(float) * 3 * mc);
  }
  std::vector<float> nxt((size_t)3 * mc, 0.f), t((size_t)3 * mc);
  for (int i = NP - 1; i >= 0; --i) {
    const float* c = &cp[(size_t)i * 9];
    for (int r = 0; r < 3; ++r)
      for (int q = 0; q < mc; ++q)
        t[(size_t)r * mc + q] = dp[((size_t)i * 3 + r) * mc + q] - (c[3 * r] * nxt[q] + c[3 * r + 1] * nxt[mc + q] + c[3 * r + 2] * nxt[2 * mc + q]);
    nxt = t;
    for (int r = 0; r < 3; ++r)
      for (int q = 0; q < mc; ++q) dmat[((size_t)i * 3 + r) * mc + q] = nxt[(size_t)r * mc + q] * cs[(size_t)i * 3 + r];
  }
}

struct Mixed {
  double theta = -1.0;       // FP32 sweep while the lane's last step exceeds it (< 0: never)
  double last = INFINITY;    // the lane's last step size in this Newton loop
  bool use32 = false;
  long steps32 = 0, steps64 = 0;
  double log_contraction = 0.0;  // sum of ln(size_k / size_{k-1}) after an FP32 step
  long contractions = 0;
};
Mixed g_mixed;

// `bordered_solve` (batch.py:595-603): delta (NP x 3) and the normalisations' step z (K)
void bordered_solve(const System& s, Vec& delta, Vec& z) {
  const int NP = s.NP, K = s.K, mc = 1 + K;
  Vec X((size_t)NP * 3 * mc);
  for (int j = 0; j < NP; ++j)
    for (int r = 0; r < 3; ++r) {
      X[((size_t)j * 3 + r) * mc] = -s.F[3 * j + r];
      for (int k = 0; k < K; ++k) X[((size_t)j * 3 + r) * mc + 1 + k] = s.U[((size_t)j * 3 + r) * K + k];
    }
  if (g_mixed.use32) block_thomas32(s, X, mc);
  else block_thomas(s, X, mc);
  Vec schur((size_t)K * K), rhs(K);
  for (int k = 0; k < K; ++k) {
    double wf = 0.0;
    for (int j = 0; j < NP; ++j) wf += s.W[(size_t)k * NP + j] * X[((size_t)j * 3) * mc];
    rhs[k] = -s.g[k] - wf;
    for (int l = 0; l < K; ++l) {
      double wu = 0.0;
      for (int j = 0; j < NP; ++j) wu += s.W[(size_t)k * NP + j] * X[((size_t)j * 3) * mc + 1 + l];
      schur[(size_t)k * K + l] = s.D[(size_t)k * K + l] - wu;
    }
  }
  lu_solve(schur.data(), rhs.data(), K, 1);
  z = rhs;
  delta.assign((size_t)NP * 3, 0.0);
  for (int j = 0; j < NP; ++j)
    for (int r = 0; r < 3; ++r) {
      double v = 0.0;
      for (int k = 0; k < K; ++k) v += X[((size_t)j * 3 + r) * mc + 1 + k] * z[k];
      delta[3 * j + r] = X[((size_t)j * 3 + r) * mc] - v;
    }
}

// `bounds` (batch.py:255-259) into full[0], full[NP + 1]
void set_bounds(const Model& m, double Vint, Vec& full) {
  const ddc_device* d = m.d;
  const double e = d->left_elec;
  full[0] = d->V0 + 0.5 * e * Vint; full[1] = d->ln_n_left; full[2] = d->ln_p_left;
  const int r = 3 * (m.NP + 1);
  full[r] = d->VL - 0.5 * e * Vint; full[r + 1] = d->ln_n_right; full[r + 2] = d->ln_p_right;
}

// `newton_step` (batch.py:759-785; solver.py:1563-1608): y (NP x 3) and logs updated, the size
Vec g_full;
double newton_step(const Model& m, Vec& y, Vec& logs, double Vint, System& s) {
  const int NP = m.NP, K = m.K;
  const double Vt = m.d->Vt, nf = m.d->n_floor;
  g_full.assign((size_t)3 * (NP + 2), 0.0);
  set_bounds(m, Vint, g_full);
  std::memcpy(&g_full[3], y.data(), sizeof(double) * 3 * NP);
  assemble(m, g_full, logs.data(), s);
  Vec delta, z;
  bordered_solve(s, delta, z);
  const double caps[3] = {CAPS[0] * Vt, CAPS[1], CAPS[2]};
  const double lognf = std::log(nf);
  double sV = 0.0, sD = 0.0, sL = 0.0;
  for (int j = 0; j < NP; ++j) {
    double step[3];
    for (int r = 0; r < 3; ++r) step[r] = clip(delta[3 * j + r], -caps[r], caps[r]);
    for (int r = 1; r < 3; ++r) {  // `density_steps` (solver.py:74-88)
      const double dd = delta[3 * j + r];
      const bool below = y[3 * j + r] < lognf;
      const bool positive = dd > -1.0;
      double in_n = positive ? std::log1p((positive && below) ? dd : 0.0) : -CAPS[1];
      in_n = clip(in_n, -FLOOR_DROP_CAP, CAPS[1]);
      if (below) step[r] = in_n;
    }
    for (int r = 0; r < 3; ++r) y[3 * j + r] = y[3 * j + r] + step[r];
    sV = nmax(sV, std::fabs(step[0]));
    for (int r = 1; r < 3; ++r) {
      const double dens = std::exp(y[3 * j + r]);
      sD = nmax(sD, std::fabs(step[r]) * (dens / (dens + nf)));
    }
  }
  for (int k = 0; k < K; ++k) {
    const double dl = clip(z[k], -ION_LOG_CAP, ION_LOG_CAP);
    logs[k] = logs[k] + dl;
    sL = nmax(sL, std::fabs(dl));
  }
  return nmax(nmax(sV / Vt, sD), sL);
}

// `current` (batch.py:302-403): the integral (or differential) terminal current at full
double current(const Model& m, const Vec& full) {
  const ddc_device* d = m.d;
  const int NP = m.NP;
  const double Vt = d->Vt, L = d->L;
  Vec V(NP + 2), n(NP + 2), p(NP + 2), R(NP + 2), Rin(NP + 2, 0.0), Rip(NP + 2, 0.0);
  for (int i = 0; i < NP + 2; ++i) {
    V[i] = full[3 * i]; n[i] = std::exp(full[3 * i + 1]); p[i] = std::exp(full[3 * i + 2]);
    double a, b;
    recombination(d, i, n[i], p[i], R[i], a, b);
  }
  if (m.any_traps) {  // `_iface_points` (solver.py:865-873)
    Vec v0(NP + 1), v1(NP + 1), v2(NP + 1), v3(NP + 1);
    for (int e = 0; e <= NP; ++e) {
      double v[5], dv[4][5];
      iface_edge(m, e, n[e], n[e + 1], p[e], p[e + 1], v, dv);
      v0[e] = v[0]; v1[e] = v[1]; v2[e] = v[2]; v3[e] = v[3];
    }
    Rin[0] = v0[0]; Rip[0] = v2[0];
    for (int k = 1; k <= NP; ++k) { Rin[k] = v1[k - 1] + v0[k]; Rip[k] = v3[k - 1] + v2[k]; }
    Rin[NP + 1] = v1[NP]; Rip[NP + 1] = v3[NP];
  }
  auto carrier = [&](double sn, const double* off, const Vec& dens, const double* mu, const Vec& Ri, Vec& Jout) {
    Vec Uc(NP + 2), Vg(NP + 2);
    for (int i = 0; i < NP + 2; ++i) { Uc[i] = R[i] + Ri[i] - d->G[i] * d->g_frac; Vg[i] = V[i] + off[i]; }
    Uc[0] = 0.0; Uc[NP + 1] = 0.0;
    Vec ev(NP + 1), int_u(NP + 1);
    for (int k = 0; k <= NP; ++k) ev[k] = std::exp(sn * Vg[k] / Vt);
    int_u[0] = 0.0;
    double acc = 0.0;
    for (int e = 0; e < NP; ++e) {
      const double dx = d->x[e + 1] - d->x[e];
      acc += 0.5 * dx * (Uc[e] + Uc[e + 1]);
      int_u[e + 1] = acc;
    }
    double single = 0.0, dbl = 0.0;
    for (int e = 0; e < NP; ++e) {
      const double dx = d->x[e + 1] - d->x[e];
      single += 0.5 * dx * (ev[e] / mu[e] + ev[e + 1] / mu[e + 1]);
      dbl += 0.5 * dx * (ev[e] * int_u[e] / mu[e] + ev[e + 1] * int_u[e + 1] / mu[e + 1]);
    }
    const double K = (Vt * (sn * dens[NP + 1] * std::exp(sn * Vg[NP + 1] / Vt) -
                            sn * dens[0] * std::exp(sn * Vg[0] / Vt)) - sn * dbl) / single;
    Vec J(NP + 1);
    double cum = 0.0;
    J[0] = Q * K;
    for (int e = 1; e <= NP; ++e) {
      cum += sn * Q * L * d->h[e] * Uc[e];
      J[e] = Q * K + cum;
    }
    if (d->curr_diff > 0.0) {
      for (int e = 0; e <= NP; ++e) {
        const double dV = sn * (Vg[e + 1] - Vg[e]) / Vt;
        double Bm, Bp, t1, t2;
        bern(-dV, m.simss, Bm, t1);
        bern(dV, m.simss, Bp, t2);
        J[e] = sn * Q * mu[e] * Vt * (dens[e + 1] * Bm - dens[e] * Bp) / (L * d->h[e]);
      }
    }
    Jout.assign(NP + 1, 0.0);
    for (int e = 0; e <= NP; ++e) {
      const double through = sn * 0.5 * Q * L * d->h[e] * (Ri[e] + Ri[e + 1]);
      Jout[e] = d->iface[e] ? J[e == 0 ? NP : e - 1] + through : J[e];
    }
  };
  Vec Jn, Jp;
  carrier(-1.0, d->offset_n, n, d->mu_n, Rin, Jn);
  carrier(1.0, d->offset_p, p, d->mu_p, Rip, Jp);
  const double sgn = -d->left_elec;
  double num = 0.0, den = 0.0;
  for (int e = 0; e <= NP; ++e) {
    num += d->h[e] * (sgn * Jn[e] + sgn * Jp[e]);
    den += d->h[e];
  }
  return num / den;
}

bool finite_state(const Vec& y, const Vec& logs) {
  for (double v : y)
    if (!std::isfinite(v)) return false;
  for (double v : logs)
    if (!std::isfinite(v)) return false;
  return true;
}

struct LoopOut {
  double J;
  bool conv;
  int it;
};

// `newton_loop` (batch.py:740-848): damped Newton until converged, max_iter or a NaN step
LoopOut newton_loop(const Model& m, Vec& y, Vec& logs, double Vint, double tol, int max_iter,
                    bool strict, System& s) {
  double sh[STALL_STEPS + 1], jh[STALL_STEPS + 1];
  for (int q = 0; q <= STALL_STEPS; ++q) { sh[q] = INFINITY; jh[q] = INFINITY; }
  int it = 0;
  bool done = false;
  Vec full((size_t)3 * (m.NP + 2));
  g_mixed.last = INFINITY;
  while (!done && it < max_iter && !std::isnan(sh[STALL_STEPS])) {
    const bool was32 = g_mixed.use32 && it > 0;
    g_mixed.use32 = g_mixed.theta >= 0.0 && !(g_mixed.last <= g_mixed.theta);
    if (g_mixed.use32) ++g_mixed.steps32;
    else ++g_mixed.steps64;
    const double size = newton_step(m, y, logs, Vint, s);
    if (was32 && g_mixed.last > 0.0 && size > 0.0 && std::isfinite(size)) {
      g_mixed.log_contraction += std::log(size / g_mixed.last);
      ++g_mixed.contractions;
    }
    g_mixed.last = size;
    set_bounds(m, Vint, full);
    std::memcpy(&full[3], y.data(), sizeof(double) * 3 * m.NP);
    const double J = current(m, full);
    for (int q = 0; q < STALL_STEPS; ++q) { sh[q] = sh[q + 1]; jh[q] = jh[q + 1]; }
    sh[STALL_STEPS] = size; jh[STALL_STEPS] = J;
    ++it;
    const double prev = sh[STALL_STEPS - 1];
    double mx = sh[0], mn = sh[1];
    for (int q = 1; q <= STALL_STEPS; ++q) mx = nmax(mx, sh[q]);
    for (int q = 2; q <= STALL_STEPS; ++q) mn = (std::isnan(mn) || std::isnan(sh[q])) ? NAN : (sh[q] < mn ? sh[q] : mn);
    const bool stalled = it > STALL_STEPS && mx < ROUND_OFF_FLOOR && mn >= 0.1 * sh[0];
    const double scale = m.d->J_scale + std::fabs(jh[STALL_STEPS]);
    double dj = 0.0;
    for (int q = 0; q <= STALL_STEPS; ++q) dj = nmax(dj, std::fabs(jh[q] - jh[STALL_STEPS]));
    const bool settled = it > STALL_STEPS && size < CURRENT_STEP_CAP && dj < CURRENT_TOL * scale;
    const bool quadratic = it > 1 && size < QUADRATIC_TOL && size < QUADRATIC_RATIO * prev;
    done = strict ? (size < tol || stalled) : (size < tol || stalled || settled || quadratic);
  }
  return {jh[STALL_STEPS], done, it};
}

// `ion_logs` (solver.py:1695-1725): the normalisations that put each slot's total into its
// region at the potential V (NP + 2)
void ion_logs(const Model& m, const Vec& V, Vec& logs) {
  logs.assign(m.K, 0.0);
  for (int k = 0; k < m.K; ++k) {
    double num = 0.0;
    for (int e = 0; e <= m.NP; ++e) {
      const double pair = m.mask(k, e + 1) * m.mask(k, e);
      const double a = m.mask(k, e + 1) * std::exp(m.sign[k] * V[e + 1] / m.d->Vt);
      const double b = m.mask(k, e) * std::exp(m.sign[k] * V[e] / m.d->Vt);
      num += 0.5 * (a + b) * pair * m.d->hL[e];
    }
    const bool has = m.totals[k] > 0.0;
    logs[k] = has ? std::log(m.totals[k] / num) : 0.0;
  }
}

// a scalar tridiagonal solve (`tridiag`, `lax.linalg.tridiagonal_solve`), rhs NP x c
void tridiag(const Vec& lo, const Vec& mid, const Vec& up, Vec& rhs, int c) {
  const int NP = (int)mid.size();
  Vec cp(NP), dp((size_t)NP * c);
  double c_prev = 0.0;
  std::vector<double> d_prev(c, 0.0);
  for (int i = 0; i < NP; ++i) {
    const double mm = mid[i] - lo[i] * c_prev;
    c_prev = up[i] / mm;
    for (int q = 0; q < c; ++q) d_prev[q] = (rhs[(size_t)i * c + q] - lo[i] * d_prev[q]) / mm;
    cp[i] = c_prev;
    for (int q = 0; q < c; ++q) dp[(size_t)i * c + q] = d_prev[q];
  }
  std::vector<double> nxt(c, 0.0);
  for (int i = NP - 1; i >= 0; --i)
    for (int q = 0; q < c; ++q) {
      nxt[q] = dp[(size_t)i * c + q] - cp[i] * nxt[q];
      rhs[(size_t)i * c + q] = nxt[q];
    }
}

// `poisson_delta` (solver.py:1757-1800) with the ions coupled: the potential's step (NP)
void poisson_delta(const Model& m, const Vec& full, Vec& step) {
  const ddc_device* d = m.d;
  const int NP = m.NP, K = m.K;
  const double Vt = d->Vt;
  Vec V(NP + 2);
  for (int i = 0; i < NP + 2; ++i) V[i] = full[3 * i];
  Vec logs;
  ion_logs(m, V, logs);
  Vec la, lc;
  point_logs(m, logs.data(), la, lc);
  Vec F(NP), mid(NP), lo(NP), up(NP), ea(NP), ec(NP);
  for (int j = 0; j < NP; ++j) {
    const int i = j + 1;
    const double n = std::exp(full[3 * i + 1]), p = std::exp(full[3 * i + 2]);
    ea[j] = m.a_mask[j] * std::exp(la[j] + V[i] / Vt);
    ec[j] = m.c_mask[j] * std::exp(lc[j] - V[i] / Vt);
    F[j] = (d->fac_l[j] * V[i - 1] + d->fac_m[j] * V[i] + d->fac_u[j] * V[i + 1] -
            Q * (n - p + d->dop[j] + m.a_fix[j] + ea[j] - m.c_fix[j] - ec[j])) * d->sP[j];
    mid[j] = (d->fac_m[j] - Q * (n + p) / Vt - Q * (ea[j] + ec[j]) / Vt) * d->sP[j];
    lo[j] = d->fac_l[j] * d->sP[j];
    up[j] = d->fac_u[j] * d->sP[j];
  }
  lo[0] = 0.0;
  up[NP - 1] = 0.0;
  Vec dV(NP);
  for (int j = 0; j < NP; ++j) dV[j] = -F[j];
  tridiag(lo, mid, up, dV, 1);
  const double cap = CAPS[0] * Vt;
  step.resize(NP);
  if (!m.mobile()) {
    for (int j = 0; j < NP; ++j) step[j] = clip(dV[j], -cap, cap);
    return;
  }
  Vec XU((size_t)NP * K);
  for (int j = 0; j < NP; ++j)
    for (int k = 0; k < K; ++k) {
      const double u = k < m.ka ? (-Q * ea[j]) * d->sP[j] : (Q * ec[j]) * d->sP[j];
      XU[(size_t)j * K + k] = u * m.mask(k, j + 1);
    }
  tridiag(lo, mid, up, XU, K);
  // the constraints at V (`ion_constraints`)
  Vec g(K), W((size_t)K * NP), Dm((size_t)K * K, 0.0);
  for (int k = 0; k < K; ++k) {
    Vec dens(NP + 2);
    for (int i = 0; i < NP + 2; ++i) dens[i] = m.mask(k, i) * std::exp(logs[k] + m.sign[k] * V[i] / Vt);
    double number = 0.0;
    for (int e = 0; e <= NP; ++e)
      number += 0.5 * (dens[e + 1] + dens[e]) * (m.mask(k, e + 1) * m.mask(k, e)) * d->hL[e];
    const bool has = m.totals[k] > 0.0;
    const double tot = has ? m.totals[k] : 1.0;
    g[k] = has ? number / tot - 1.0 : 0.0;
    for (int j = 0; j < NP; ++j) {
      const double pl = m.mask(k, j + 1) * m.mask(k, j) * d->hL[j];
      const double pr = m.mask(k, j + 2) * m.mask(k, j + 1) * d->hL[j + 1];
      W[(size_t)k * NP + j] = has ? 0.5 * (pl + pr) * dens[j + 1] * m.sign[k] / Vt / tot : 0.0;
    }
    Dm[(size_t)k * K + k] = (has ? number / tot : 0.0) + (has ? 0.0 : 1.0);
  }
  Vec S((size_t)K * K), r(K);
  for (int k = 0; k < K; ++k) {
    double wv = 0.0;
    for (int j = 0; j < NP; ++j) wv += W[(size_t)k * NP + j] * dV[j];
    r[k] = -g[k] - wv;
    for (int l = 0; l < K; ++l) {
      double wu = 0.0;
      for (int j = 0; j < NP; ++j) wu += W[(size_t)k * NP + j] * XU[(size_t)j * K + l];
      S[(size_t)k * K + l] = Dm[(size_t)k * K + l] - wu;
    }
  }
  lu_solve(S.data(), r.data(), K, 1);
  double mx = 0.0;
  for (int j = 0; j < NP; ++j) {
    double v = 0.0;
    for (int k = 0; k < K; ++k) v += XU[(size_t)j * K + k] * r[k];
    step[j] = dV[j] - v;
    mx = nmax(mx, std::fabs(step[j]));
  }
  mx = mx / Vt;
  const double f = mx > 0.0 ? std::fmin(std::log1p(mx), CAPS[0]) / mx : 1.0;
  for (int j = 0; j < NP; ++j) step[j] = step[j] * f;
}

// `poisson_solve` (batch.py:486-503)
void poisson_solve(const Model& m, Vec& y, double Vint, int max_iter) {
  double size = INFINITY;
  int it = 0;
  Vec full((size_t)3 * (m.NP + 2)), dV;
  while (size > 1e-8 && it < max_iter) {
    set_bounds(m, Vint, full);
    std::memcpy(&full[3], y.data(), sizeof(double) * 3 * m.NP);
    poisson_delta(m, full, dV);
    size = 0.0;
    for (int j = 0; j < m.NP; ++j) {
      const double shift = dV[j] / m.d->Vt;
      y[3 * j] = y[3 * j] + dV[j];
      y[3 * j + 1] = y[3 * j + 1] + shift;
      y[3 * j + 2] = y[3 * j + 2] + -shift;
      size = nmax(size, std::fabs(shift));
    }
    ++it;
  }
}

// `initial` (batch.py:276-299) at interior points
void initial(const Model& m, double Vint, Vec& y) {
  const ddc_device* d = m.d;
  y.assign((size_t)3 * m.NP, 0.0);
  const double e = d->left_elec;
  for (int j = 0; j < m.NP; ++j) {
    const int i = j + 1;
    const double x = d->x[i];
    const double V = d->V0 + 0.5 * e * Vint + x * (d->VL - d->V0 - e * Vint) / d->L;
    const double EF = d->W_L - x * (d->W_L - d->W_R) / d->L;
    const double ln_n = std::log(d->N_c[i]) - (EF - d->E_c[i]) / d->Vt;
    y[3 * j] = V; y[3 * j + 1] = ln_n; y[3 * j + 2] = 2.0 * std::log(d->ni[i]) - ln_n;
  }
}

void full_V(const Model& m, const Vec& y, double Vint, Vec& V) {
  V.resize(m.NP + 2);
  const double e = m.d->left_elec;
  V[0] = m.d->V0 + 0.5 * e * Vint;
  V[m.NP + 1] = m.d->VL - 0.5 * e * Vint;
  for (int j = 0; j < m.NP; ++j) V[j + 1] = y[3 * j];
}

// `start` (batch.py:875-934): Poisson, then Newton at `first`, through the ion-density stages
// where that fails on a device with mobile ions
bool start(Model& m, double first, double tol, int start_iter, bool strict, Vec& y, Vec& logs, System& s) {
  Vec y0;
  initial(m, first, y0);
  poisson_solve(m, y0, first, start_iter);
  Vec V;
  full_V(m, y0, first, V);
  ion_logs(m, V, logs);
  y = y0;
  Vec y_f = y0, logs_f = logs;
  const LoopOut f = newton_loop(m, y_f, logs_f, first, tol, start_iter, strict, s);
  const bool done = f.conv || !m.mobile();
  bool staged = false;
  Vec y_c = y0, logs_c = logs;
  if (!done) {
    const Vec a_fix0 = m.a_fix, c_fix0 = m.c_fix, tot0 = m.totals;
    double before = 1.0;
    bool ok_c = true;
    for (double share : STAGES) {  // `_scaled` (solver.py:2012-2015)
      for (int j = 0; j < m.NP; ++j) { m.a_fix[j] = a_fix0[j] * share; m.c_fix[j] = c_fix0[j] * share; }
      for (int k = 0; k < m.K; ++k) m.totals[k] = tot0[k] * share;
      for (int k = 0; k < m.K; ++k) logs_c[k] = logs_c[k] + std::log(share / before);
      Vec y_k = y_c, logs_k = logs_c;
      ok_c = newton_loop(m, y_k, logs_k, first, tol, start_iter, strict, s).conv;
      if (finite_state(y_k, logs_k)) { y_c = y_k; logs_c = logs_k; }
      before = share;
    }
    m.a_fix = a_fix0; m.c_fix = c_fix0; m.totals = tot0;
    staged = ok_c;
  }
  if (staged) { y = y_c; logs = logs_c; }
  else if (finite_state(y_f, logs_f)) { y = y_f; logs = logs_f; }
  return f.conv || staged;
}

// `freeze` (batch.py:859-872): the mobile ions of y as fixed densities
void freeze(Model& m, const Vec& y, const Vec& logs) {
  Vec la, lc;
  point_logs(m, logs.data(), la, lc);
  for (int j = 0; j < m.NP; ++j) {
    const double V = y[3 * j];
    m.a_fix[j] = m.a_fix[j] + m.a_mask[j] * std::exp(la[j] + V / m.d->Vt);
    m.c_fix[j] = m.c_fix[j] + m.c_mask[j] * std::exp(lc[j] - V / m.d->Vt);
    m.a_mask[j] = 0.0; m.c_mask[j] = 0.0;
  }
  std::fill(m.masks.begin(), m.masks.end(), 0.0);
  std::fill(m.totals.begin(), m.totals.end(), 0.0);
}

// `solve_one` (batch.py:937-1006): start, pre-bias (ions frozen after it where `fixIons`), the
// scan up from the pre-bias and down from it again, each voltage from the last two converged
// solutions extrapolated; voltages ascending
void solve_one(const ddc_device* d, bool simss, const double* vs, int nv, double tol, int max_iter,
               int start_iter, bool strict, double* J, uint8_t* ok, int32_t* its) {
  Model m(d, simss);
  System s;
  s.size(m.NP, m.K);
  const double first = d->pre_cond > 0.0 ? d->V_pre : vs[0];
  Vec y, logs;
  const bool solved = start(m, first, tol, start_iter, strict, y, logs, s);
  bool pre_ok = true;
  if (!solved) pre_ok = newton_loop(m, y, logs, first, tol, start_iter, strict, s).conv;
  const bool frozen = d->pre_cond > 0.0 && d->fix_ions > 0.0;
  if (frozen) {
    freeze(m, y, logs);
  } else {
    pre_ok = true;
  }
  int below = 0;
  while (below < nv && vs[below] < first) ++below;
  const double caps[3] = {CAPS[0] * d->Vt, CAPS[1], CAPS[2]};
  Vec yc = y, lc = logs, yp = y, lp = logs;
  double V_last = first, V_before = first;
  for (int k = 0; k < nv; ++k) {
    if (k == nv - below) {  // the scan turns: back to the pre-bias solution
      yc = y; lc = logs; yp = y; lp = logs; V_last = first; V_before = first;
    }
    const int idx = k < nv - below ? below + k : nv - 1 - k;
    const double Vint = vs[idx];
    const double ratio = V_last != V_before ? (Vint - V_last) / (V_last - V_before) : 0.0;
    Vec guess(yc.size()), lguess(lc.size());
    for (size_t q = 0; q < yc.size(); ++q) {
      const double c = caps[q % 3];
      guess[q] = yc[q] + clip(ratio * (yc[q] - yp[q]), -c, c);
    }
    for (size_t q = 0; q < lc.size(); ++q)
      lguess[q] = lc[q] + clip(ratio * (lc[q] - lp[q]), -ION_LOG_CAP, ION_LOG_CAP);
    const LoopOut o = newton_loop(m, guess, lguess, Vint, tol, max_iter, strict, s);
    if (o.conv && finite_state(guess, lguess)) {
      yp = yc; lp = lc; yc = guess; lc = lguess; V_before = V_last; V_last = Vint;
    }
    J[idx] = o.J;
    ok[idx] = (o.conv && pre_ok) ? 1 : 0;
    its[idx] = o.it;
  }
}

}  // namespace

// `solve_batch` (batch.py:1136-1162, `_passes` 1194-1208) for one device: J, converged and
// iterations at `voltages` in the caller's order, the shunt's current added. Two passes: every
// voltage with `first_max_iter` Newton steps, then, if any missed it, the whole device again with
// `max_iter`.
int ddc_solve_batch(const ddc_device* dev, const double* voltages, int nv, double tol,
                    int max_iter, int first_max_iter, int simss, double* J, uint8_t* converged,
                    int32_t* iterations) {
  if (!dev || !voltages || nv < 1 || !J || !converged || !iterations || dev->NP < 3) return 1;
  std::vector<int> order(nv);
  for (int k = 0; k < nv; ++k) order[k] = k;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return voltages[a] < voltages[b]; });
  Vec vs(nv), Js(nv);
  std::vector<uint8_t> oks(nv);
  std::vector<int32_t> itss(nv);
  for (int k = 0; k < nv; ++k) vs[k] = voltages[order[k]];
  const bool one_pass = first_max_iter <= 0 || first_max_iter >= max_iter;
  solve_one(dev, simss != 0, vs.data(), nv, tol, one_pass ? max_iter : first_max_iter, max_iter,
            false, Js.data(), oks.data(), itss.data());
  bool all = true;
  for (int k = 0; k < nv; ++k) all = all && oks[k];
  if (!one_pass && !all)
    solve_one(dev, simss != 0, vs.data(), nv, tol, max_iter, max_iter, false, Js.data(), oks.data(),
              itss.data());
  for (int k = 0; k < nv; ++k) {
    J[order[k]] = Js[k] + dev->G_shunt * vs[k];
    converged[order[k]] = oks[k];
    iterations[order[k]] = itss[k];
  }
  return 0;
}

// jaxdd's solve_batch with the per-lane mixed-precision sweep (`Mixed`): an FP32 sweep while the
// lane's last Newton step in scaled units exceeds `theta`, FP64 for the finish. stats[0..3]: the
// steps with an FP32 sweep, those with an FP64 one, the geometric mean of the step-size ratio
// after an FP32 step, the number of such ratios. One pass at max_iter.
extern "C" int ddc_solve_batch_mixed(const ddc_device* dev, const double* voltages, int nv,
                                     double tol, int max_iter, int simss, double theta,
                                     double* J, uint8_t* converged, int32_t* iterations,
                                     double* stats) {
  g_mixed = Mixed();
  g_mixed.theta = theta;
  const int st = ddc_solve_batch(dev, voltages, nv, tol, max_iter, 0, simss, J, converged,
                                 iterations);
  if (stats) {
    stats[0] = (double)g_mixed.steps32;
    stats[1] = (double)g_mixed.steps64;
    stats[2] = g_mixed.contractions ? std::exp(g_mixed.log_contraction / g_mixed.contractions) : NAN;
    stats[3] = (double)g_mixed.contractions;
  }
  g_mixed = Mixed();
  return st;
}
