// Batched steady-state drift-diffusion J-V solve for sm_100a: one persistent launch, two
// threads per device (a "pair" of adjacent lanes), every array lane-interleaved (dd_layout.h).
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
//  * The block tridiagonal system is solved by a twisted (two-sided) factorisation: half 0 of a
//    pair eliminates rows 1..mid-1 downwards while half 1 eliminates rows NP..mid+1 upwards;
//    they meet at row mid (one 3x3 solve with the "twisted pivot" B - A c' - C a''), then each
//    back-substitutes its own half. The serial chain per thread is half the grid and twice the
//    threads are in flight. Each row is assembled in registers as it is eliminated (each
//    interval's fluxes once); only c' (or a'') and d' go to memory.
//  * The ions' border is carried along both eliminations (w = U^-T W and the sums w^T d'), so
//    its K x K Schur complement is solved at the meeting row and one back substitution with the
//    right-hand side d'_F - d'_U z gives the bordered step directly.
//  * The back substitution damps (`density_steps`), updates the state in place, measures the
//    step, and accumulates the terminal current: half 0 right to left with suffix sums, half 1
//    left to right with prefix sums, combined exactly at the end (no pass of its own).
//  * Each device runs its own program (start, pre-bias, scan) as a state machine; every loop
//    iteration takes one Newton (or Poisson) step at that device's own voltage. Devices never
//    wait for another device's voltages, so jaxdd's two passes (first_max_iter, then
//    stragglers, batch.py:1194-1208) collapse into one pass at max_iter with the same results.
//    The pair takes every decision on half 0's values (broadcast by warp shuffles), so the two
//    threads never part ways; they exchange data only through shuffles.
//  * Every loop is bounded (caps on Poisson and Newton steps, voltages, stages): the kernel
//    always terminates.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <utility>
#include <vector>

// With DD_OUTLINE_MATH 1 the sweeps' expm1 (the Bernoulli function), with 2 also their exp and
// log1p, have one out-of-line copy that every call site shares instead of a copy inlined at each
// site: the step's code is large enough that instruction fetch, not arithmetic, limits how often
// a warp issues.
#if defined(DD_OUTLINE_MATH) && DD_OUTLINE_MATH >= 1
__device__ __noinline__ double dd_expm1_shared(double x) { return expm1(x); }
#define DD_EXPM1(x) dd_expm1_shared(x)
#endif
#if defined(DD_OUTLINE_MATH) && DD_OUTLINE_MATH >= 2
__device__ __noinline__ double dd_exp_shared(double x) { return exp(x); }
__device__ __noinline__ double dd_log1p_shared(double x) { return log1p(x); }
#define DD_EXP(x) dd_exp_shared(x)
#define DD_LOG1P(x) dd_log1p_shared(x)
#endif

#include "dd_launch.h"
#include "dd_layout.h"
#include "dd_physics.cuh"
#include "../../include/jaxdd_b200.h"

namespace dd {

__device__ __constant__ double c_stage_share[4] = {1.0 / 64, 1.0 / 16, 1.0 / 4, 1.0};

// Threads per block of the solve (two per device, the pairs adjacent lanes of a warp). One warp
// a block spreads a batch's warps over the 148 SMs more evenly than two (at the drawn J-V curves' 16384
// devices: at most 7 warps on an SM instead of 8; 2.2 % faster measured).
#ifndef DD_SOLVE_BLOCK
#define DD_SOLVE_BLOCK 32
#endif

// ------------------------------------------------------------------------------------ prefetch

// A hint to bring one line into L1 ahead of its use: each node's record and state are read from
// HBM one after another along the sweep, and too few warps run per SM to hide that latency.
// The sweeps ask for the node DD_PREFETCH_AHEAD positions ahead of the one they work on.
// Measured on the drawn J-V curves (16384 devices, NP 400, 61 V): one position ahead 20,644 curves/s, two 19,976, four 17,715 (L1 is
// too small for more nodes' lines per warp); L2 hints further ahead on top of it made it slower.
#ifndef DD_PREFETCH_AHEAD
#define DD_PREFETCH_AHEAD 1
#endif
__device__ __forceinline__ void prefetch_line(const double* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// Node k's whole static record and its state (k within the device's nodes).
__device__ __forceinline__ void prefetch_node(const Lane& L, int k) {
  if (k < 0 || k > L.NP + 1) return;
#pragma unroll
  for (int f = 0; f < DD_NF; ++f) prefetch_line(L.S + ((size_t)k * DD_NF + f) * L.Bp + L.l);
#pragma unroll
  for (int c = 0; c < 3; ++c) prefetch_line(L.y(0, k, c));
}

// Node k's sweep record (c', d') for the back substitution.
__device__ __forceinline__ void prefetch_cd(const Lane& L, int k) {
  if (k < 1 || k > L.NP) return;
  for (int f = 0; f < L.ncd; ++f) prefetch_line(L.cd(k, f));
}

// Node k's iterate (the state the forward sweep starts from, the back substitution updates).
__device__ __forceinline__ void prefetch_state(const Lane& L, int k) {
  if (k < 0 || k > L.NP + 1) return;
#pragma unroll
  for (int c = 0; c < 3; ++c) prefetch_line(L.y(0, k, c));
}

// ------------------------------------------------------------------------------------ staging
//
// The sweeps read each node's static record (DD_NF words) from a ring of three records in shared
// memory instead of from global memory field by field where each is used. A record is copied in
// by cp.async (8 bytes a thread, every thread its own lane's words: a warp's copy of one field is
// 16 consecutive words of each of two nodes) two positions before the sweep reaches it and waited
// for one position before, so the copy's latency passes behind a whole position's arithmetic.
// Ring slot = position mod 3; the block's ring is [slot][field][thread], each thread owning one
// column, so a warp's read of one field is 32 consecutive words.
constexpr int RING = 3;

// A lane whose static record reads come from the ring: the positions the sweep is at (p and
// p + 1) must be staged and waited for.
template <int BS>
struct Staged : Lane {
  double* ring;  // this thread's column of the block's ring (BS threads a block)
  __device__ __forceinline__ int pos(int k) const { return half == 0 ? k : NP + 1 - k; }
  __device__ __forceinline__ double st(int k, int f) const {
    return ring[((pos(k) % RING) * DD_NF + f) * BS];
  }
  __device__ __forceinline__ double afix(int k) const {
    return frozen ? FX[((size_t)k * 2) * Bp + l] : share * st(k, S_AFIX);
  }
  __device__ __forceinline__ double cfix(int k) const {
    return frozen ? FX[((size_t)k * 2 + 1) * Bp + l] : share * st(k, S_CFIX);
  }
};

// Copy position p's record (node p of half 0, NP + 1 - p of half 1) into its ring slot as one
// commit group; an empty group when p is outside 0 .. last, so that every position commits one.
template <int BS>
__device__ __forceinline__ void stage(const Staged<BS>& R, int p, int last) {
  if (p >= 0 && p <= last) {
    const int k = R.half == 0 ? p : R.NP + 1 - p;
    const double* src = R.S + (size_t)k * DD_NF * R.Bp + R.l;
    const unsigned dst = (unsigned)__cvta_generic_to_shared(R.ring + (p % RING) * DD_NF * BS);
#pragma unroll
    for (int f = 0; f < DD_NF; ++f)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst + f * BS * 8),
                   "l"(src + (size_t)f * R.Bp)
                   : "memory");
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}
// Every staged position but the newest is in the ring.
__device__ __forceinline__ void staged_all_but_newest() {
  asm volatile("cp.async.wait_group 1;" ::: "memory");
}
// Every staged position is in the ring (no copy into it is left in flight).
__device__ __forceinline__ void staged_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// ------------------------------------------------------------------------------------ pair

__device__ __forceinline__ double xchg(const Lane& L, double v) {
  return __shfl_xor_sync(L.mask, v, 1);
}
__device__ __forceinline__ int xchgi(const Lane& L, int v) { return __shfl_xor_sync(L.mask, v, 1); }
__device__ __forceinline__ double bcast(const Lane& L, double v) {
  return __shfl_sync(L.mask, v, L.base);
}
__device__ __forceinline__ int bcasti(const Lane& L, int v) { return __shfl_sync(L.mask, v, L.base); }

// ------------------------------------------------------------------------------------ advance

// How the first forward pass of a voltage makes its start from the carried solutions
// (`_solve_one`'s scan body, batch.py:964-1004): buffers 0 iterate, 1 carry, 2 previous carry,
// 3 the pre-bias solution. Only the thread that owns node k calls this for k.
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
      s[c] = ratio != 0.0 ? base + clipd(ratio * (base - prev), -cap[c], cap[c]) : base;
      *L.y(0, k, c) = s[c];
    }
  }
  P.V = s[0]; P.lnn = s[1]; P.lnp = s[2];
}

// The elimination carried along one direction of the twisted sweep. Going down (half 0) a row
// reads A x_{i-1} + B x_i + C x_{i+1} = r with x_{i-1} = d' - c' x_i already known in terms of
// x_i: X = A couples to the eliminated side, Y = C to the rest, and c'_i = M^-1 C,
// d'_i = M^-1 (r - A d'), M = B - A c'. Going up (half 1) the same with X = C, Y = A (x_i =
// d'' - a'' x_{i-1}). Beside them w (the border W carried through the sweep, w_i = W_i - c'^T
// w_{i-1}) and the sums w^T d', so that W^T x over this half is known without x.
template <int K>
struct Carry {
  double c[9];         // c' (or a'')
  double dF[3];        // d' of the residual column
  double dU[3][K];     // d' of the ion columns
  double w[3][K];      // w
  double S[K][K];      // sum w^T d'_U
  double s[K];         // sum w^T d'_F
  double num[K];       // the slots' ion numbers over this half's intervals

  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int j = 0; j < 9; ++j) c[j] = 0.0;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      dF[r] = 0.0;
#pragma unroll
      for (int k = 0; k < K; ++k) { dU[r][k] = 0.0; w[r][k] = 0.0; }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      s[k] = 0.0; num[k] = 0.0;
#pragma unroll
      for (int j = 0; j < K; ++j) S[k][j] = 0.0;
    }
  }

  __device__ __forceinline__ void eliminate(const double (&X)[3][3], const double (&B)[3][3],
                                            const double (&Y)[3][3], const double (&rhs)[3],
                                            const double (&U0)[K], const double (&W)[K]) {
    double M[3][3], Mi[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int q = 0; q < 3; ++q)
        M[r][q] = B[r][q] - (X[r][0] * c[q] + X[r][1] * c[3 + q] + X[r][2] * c[6 + q]);
    inv3(M, Mi);
    double wn[3][K];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int k = 0; k < K; ++k)
        wn[r][k] = (r == 0 ? W[k] : 0.0) - (c[0 + r] * w[0][k] + c[3 + r] * w[1][k] + c[6 + r] * w[2][k]);
    double tF[3], tU[3][K];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      tF[r] = rhs[r] - (X[r][0] * dF[0] + X[r][1] * dF[1] + X[r][2] * dF[2]);
#pragma unroll
      for (int k = 0; k < K; ++k)
        tU[r][k] = (r == 0 ? U0[k] : 0.0) - (X[r][0] * dU[0][k] + X[r][1] * dU[1][k] + X[r][2] * dU[2][k]);
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      dF[r] = Mi[r][0] * tF[0] + Mi[r][1] * tF[1] + Mi[r][2] * tF[2];
#pragma unroll
      for (int k = 0; k < K; ++k) dU[r][k] = Mi[r][0] * tU[0][k] + Mi[r][1] * tU[1][k] + Mi[r][2] * tU[2][k];
    }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int q = 0; q < 3; ++q)
        c[r * 3 + q] = Mi[r][0] * Y[0][q] + Mi[r][1] * Y[1][q] + Mi[r][2] * Y[2][q];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int k = 0; k < K; ++k) w[r][k] = wn[r][k];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      s[k] += w[0][k] * dF[0] + w[1][k] * dF[1] + w[2][k] * dF[2];
#pragma unroll
      for (int j = 0; j < K; ++j) S[k][j] += w[0][k] * dU[0][j] + w[1][k] * dU[1][j] + w[2][k] * dU[2][j];
    }
  }

  __device__ __forceinline__ void store(const Lane& L, int i) const {
#pragma unroll
    for (int j = 0; j < 9; ++j) *L.cd(i, j) = c[j];
#pragma unroll
    for (int r = 0; r < 3; ++r) *L.cd(i, 9 + r) = dF[r];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int k = 0; k < K; ++k) *L.cd(i, 12 + r * K + k) = dU[r][k];
  }

  // half 1 hands its carry to half 0 at the meeting row
  __device__ __forceinline__ void exchange(const Lane& L) {
#pragma unroll
    for (int j = 0; j < 9; ++j) c[j] = xchg(L, c[j]);
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      dF[r] = xchg(L, dF[r]);
#pragma unroll
      for (int k = 0; k < K; ++k) { dU[r][k] = xchg(L, dU[r][k]); w[r][k] = xchg(L, w[r][k]); }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      s[k] = xchg(L, s[k]); num[k] = xchg(L, num[k]);
#pragma unroll
      for (int j = 0; j < K; ++j) S[k][j] = xchg(L, S[k][j]);
    }
  }
};

// Newton's damping of one point (the caps and `density_steps`, solver.py:74-88), its new state
// and its contribution to the step's size.
__device__ __forceinline__ void damp(const Lane& L, const double (&x)[3], const Pt& old, Pt& nw,
                                     double& size, bool& finite) {
  const double sV = clipd(x[0], -CAP_V * L.Vt, CAP_V * L.Vt);
  double sd[2];
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const double yy = s == 0 ? old.lnn : old.lnp;
    const double d = x[1 + s];
    const bool below = yy < L.lognf;
    const bool pos = d > -1.0;
    double in_n = pos ? DD_LOG1P(below ? d : 0.0) : -CAP_LN;
    in_n = clipd(in_n, -FLOOR_DROP_CAP, CAP_LN);
    sd[s] = below ? in_n : clipd(d, -CAP_LN, CAP_LN);
  }
  nw.V = old.V + sV; nw.lnn = old.lnn + sd[0]; nw.lnp = old.lnp + sd[1];
  nw.n = DD_EXP(nw.lnn); nw.p = DD_EXP(nw.lnp);
  size = nanmax(size, fabs(sV) * L.iVt);
  size = nanmax(size, fabs(sd[0]) * (nw.n / (nw.n + L.nfloor)));
  size = nanmax(size, fabs(sd[1]) * (nw.p / (nw.p + L.nfloor)));
  finite = finite && isfinite(nw.V) && isfinite(nw.lnn) && isfinite(nw.lnp);
}

// ------------------------------------------------------------------------------------ current
//
// The terminal current (`_current_parts`, batch.py:316-403, steady state), accumulated over the
// new state in the back substitution, half 0 right to left over its points 0..mid and intervals
// 0..mid, half 1 left to right over mid+1..NP. For each carrier (electrons sn = -1, holes
// sn = +1), with U_k = R_k + R_int,k - G_k g (0 on the contacts), q_k = exp(sn Vg_k / V_T)/mu_k,
// c_k = (dx_{k-1} + dx_k)/2 and the trapezoids a_k = dx_k (U_k + U_{k+1})/2, jaxdd's
//   single = sum_k c_k q_k,   double = sum_k c_k q_k int_u_k,  int_u_k = sum_{e<k} a_e,
//   sum_e h_e J_e = qK H + sum_{k>=1} b_k Hs_k - sum_{interfaces e} h_e (b_e - t_e),
// with b_k = sn q L h_k U_k, Hs_k = sum_{e>=k} h_e and t_e the current through interval e's
// traps (an interface's J is the one before it plus t_e), are rewritten with suffix sums
// (double = A single - sum c q T, T_k = sum_{e>=k} a_e, A = T_0), so that each half needs only
// its own partial sums and the other half's totals. The differential form sums the intervals'
// Scharfetter-Gummel fluxes, an interface again taking the interval before it plus t_e.
struct CurPart {
  double single[2], cq[2], A[2], bH[2], Bs[2], corr[2];
  double H, dtot;

  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int s = 0; s < 2; ++s) { single[s] = cq[s] = A[s] = bH[s] = Bs[s] = corr[s] = 0.0; }
    H = 0.0; dtot = 0.0;
  }
  __device__ __forceinline__ void exchange(const Lane& L) {
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      single[s] = xchg(L, single[s]); cq[s] = xchg(L, cq[s]); A[s] = xchg(L, A[s]);
      bH[s] = xchg(L, bH[s]); Bs[s] = xchg(L, Bs[s]); corr[s] = xchg(L, corr[s]);
    }
    H = xchg(L, H); dtot = xchg(L, dtot);
  }
};

__device__ __forceinline__ double sg_flux(const Lane& L, int s, const Pt& a, const Pt& b,
                                          double mu, double h) {
  const double sn = s == 0 ? -1.0 : 1.0;
  const double Vga = a.V + (s == 0 ? a.offn : a.offp);
  const double Vgb = b.V + (s == 0 ? b.offn : b.offp);
  double Bf, Bb, d1, d2;
  bern_pair(sn * (Vgb - Vga) * L.iVt, L.simss, Bf, Bb, d1, d2);
  const double da = s == 0 ? a.n : a.p, db = s == 0 ? b.n : b.p;
  return sn * Q * mu * L.Vt * (db * Bb - da * Bf) / (L.L * h);
}

// ------------------------------------------------------------------------------------ Newton step

// Word j < 30 + 2K of the meeting row's record (its right-hand side, A, B, C, ion columns and
// border), held between half 0's assembly of the row and the solve at the meeting: the sweep
// records of node 0 (a contact) and of node mid (the meeting row is not eliminated), which no
// elimination writes; 2 (12 + 3K) >= 30 + 2K words.
__device__ __forceinline__ double* meet_word(const Lane& L, int j) {
  return j < L.ncd ? L.cd(0, j) : L.cd(L.mid, j - L.ncd);
}

struct StepOut {
  double size;
  double J;
  bool finite;
};

// One Newton step of a device, both threads of its pair (or, with `noise`, the round-off step
// of `_noise_step`, solver.py:1728-1751, which leaves the state as it is). Returns the same
// size, current and finiteness in both threads.
//
// Both halves run the same instructions in a mirrored frame: position p = 1 .. nown of a half
// is node p (half 0) or node NP + 1 - p (half 1), p = 0 its contact, p = nown its boundary
// point (mid, or mid + 1) and p = nown + 1 the other half's. Half 0 assembles the meeting row
// mid at p = nown instead of eliminating it.
template <int K, int BS>
__device__ StepOut newton_step(Lane& L, double Vint, double* logs, int adv, double ratio,
                               bool noise, double* ring) {
  const int NP = L.NP, m = L.mid;
  const bool top = L.half == 0;
  const bool mir = !top;
  const int nown = top ? m : NP - m;
  // position -> node; the interval between positions p and p + 1 -> its physical index
#define NODE(p) (top ? (p) : NP + 1 - (p))
#define EDGE(p) (top ? (p) : NP - (p))
  // the boundary points: each half makes its own start there (load_state writes it to the
  // iterate, where it is read again when needed) and hands the state to the other half, which
  // keeps only (V, ln n, ln p) of it and fills in the rest where it uses it
  double xb[3];
  {
    Pt t;
    load_state(L, NODE(nown), adv, ratio, t);
    xb[0] = xchg(L, t.V); xb[1] = xchg(L, t.lnn); xb[2] = xchg(L, t.lnp);
  }
  // the sweeps' static records from the ring: positions 0 (the contact) .. nown + 1 (the other
  // half's boundary point); 0 and 1 waited for, 2 on its way
  Staged<BS> R;
  static_cast<Lane&>(R) = L;
  R.ring = ring;
  const int last = nown + 1;
  stage(R, 0, last);
  stage(R, 1, last);
  stage(R, 2, last);
  staged_all_but_newest();
  auto own_boundary = [&](Pt& P) {
    P.V = *L.y(0, NODE(nown), 0); P.lnn = *L.y(0, NODE(nown), 1); P.lnp = *L.y(0, NODE(nown), 2);
    pt_fill_k<K>(R, P, NODE(nown), logs);
  };
  auto other_boundary = [&](Pt& P) {
    P.V = xb[0]; P.lnn = xb[1]; P.lnp = xb[2];
    pt_fill_k<K>(R, P, NODE(nown + 1), logs);
  };

  Carry<K> cr;
  cr.zero();
  {
    Pt pm, pc, pn;
    contact(L, top ? 0 : 1, Vint, pm);
    pt_fill_k<K>(R, pm, NODE(0), logs);
    if (nown == 1) own_boundary(pc);
    else { load_state(L, NODE(1), adv, ratio, pc); pt_fill_k<K>(R, pc, NODE(1), logs); }
    Flux el;
    int e = EDGE(0);
    double h_m = R.st(e, S_H);
    flux(L, pm, pc, R.st(e, S_MUN), R.st(e, S_MUP), el);
    ion_edge<K>(L, pm, pc, h_m * L.L, cr.num);
    int ifk_m = (int)R.st(e, S_IFK);
    for (int p = 1; p <= nown; ++p) {
      stage(R, p + 2, last);
      if (p + 2 <= last) prefetch_state(L, NODE(p + 2));
      staged_all_but_newest();  // positions p and p + 1
      if (p + 1 == nown) own_boundary(pn);
      else if (p == nown) other_boundary(pn);
      else { load_state(L, NODE(p + 1), adv, ratio, pn); pt_fill_k<K>(R, pn, NODE(p + 1), logs); }
      e = EDGE(p);
      const double h_i = R.st(e, S_H);
      const int ifk_i = (int)R.st(e, S_IFK);
      Flux er;
      flux(L, pc, pn, R.st(e, S_MUN), R.st(e, S_MUP), er);
      if (p < nown || top) ion_edge<K>(L, pc, pn, h_i * L.L, cr.num);  // interval mid is half 0's
      double A[3][3], Bm[3][3], Cm[3][3], rhs[3], U0[K], W[K];
      assemble_row<K>(R, NODE(p), pm, pc, pn, el, er, h_m, h_i, ifk_m, ifk_i, noise, mir, A, Bm,
                      Cm, rhs, U0, W);
      if (p < nown || !top) {
        cr.eliminate(A, Bm, Cm, rhs, U0, W);
        cr.store(L, NODE(p));
      } else {
        // the meeting row waits in memory until both halves are through (kept in registers it
        // would hold them over the whole loop)
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          *meet_word(L, r) = rhs[r];
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            *meet_word(L, 3 + 3 * r + q) = A[r][q];
            *meet_word(L, 12 + 3 * r + q) = Bm[r][q];
            *meet_word(L, 21 + 3 * r + q) = Cm[r][q];
          }
        }
#pragma unroll
        for (int k = 0; k < K; ++k) { *meet_word(L, 30 + k) = U0[k]; *meet_word(L, 30 + K + k) = W[k]; }
      }
      pm = pc; pc = pn; el = er; h_m = h_i; ifk_m = ifk_i;
    }
  }
  // ---------------------------------------------------------------- the meeting row mid
  Carry<K> other = cr;
  other.exchange(L);  // half 0 now holds half 1's carry (a''_{mid+1}, d''_{mid+1}, ...)
  double z[K], xm[3];
#pragma unroll
  for (int k = 0; k < K; ++k) z[k] = 0.0;
  if (top) {
    double Am[3][3], Bmm[3][3], Cmm[3][3], rm[3], Um[K], Wm[K];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      rm[r] = *meet_word(L, r);
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        Am[r][q] = *meet_word(L, 3 + 3 * r + q);
        Bmm[r][q] = *meet_word(L, 12 + 3 * r + q);
        Cmm[r][q] = *meet_word(L, 21 + 3 * r + q);
      }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) { Um[k] = *meet_word(L, 30 + k); Wm[k] = *meet_word(L, 30 + K + k); }
    // gamma x_mid = [r | U]_mid - A d'_{mid-1} - C d''_{mid+1}, gamma = B - A c' - C a''
    double G[3][3], Gi[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int q = 0; q < 3; ++q)
        G[r][q] = Bmm[r][q] - (Am[r][0] * cr.c[q] + Am[r][1] * cr.c[3 + q] + Am[r][2] * cr.c[6 + q]) -
                  (Cmm[r][0] * other.c[q] + Cmm[r][1] * other.c[3 + q] + Cmm[r][2] * other.c[6 + q]);
    inv3(G, Gi);
    double RF[3], RU[3][K];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      RF[r] = rm[r] - (Am[r][0] * cr.dF[0] + Am[r][1] * cr.dF[1] + Am[r][2] * cr.dF[2]) -
              (Cmm[r][0] * other.dF[0] + Cmm[r][1] * other.dF[1] + Cmm[r][2] * other.dF[2]);
#pragma unroll
      for (int k = 0; k < K; ++k)
        RU[r][k] = (r == 0 ? Um[k] : 0.0) -
                   (Am[r][0] * cr.dU[0][k] + Am[r][1] * cr.dU[1][k] + Am[r][2] * cr.dU[2][k]) -
                   (Cmm[r][0] * other.dU[0][k] + Cmm[r][1] * other.dU[1][k] + Cmm[r][2] * other.dU[2][k]);
    }
    double XF[3], XU[3][K];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      XF[r] = Gi[r][0] * RF[0] + Gi[r][1] * RF[1] + Gi[r][2] * RF[2];
#pragma unroll
      for (int k = 0; k < K; ++k) XU[r][k] = Gi[r][0] * RU[0][k] + Gi[r][1] * RU[1][k] + Gi[r][2] * RU[2][k];
    }
    if (!noise) {
      // W^T x = both halves' sums + (W_mid - c'^T w' - a''^T w'')^T x_mid
      double wh[3][K];
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < K; ++k)
          wh[r][k] = (r == 0 ? Wm[k] : 0.0) -
                     (cr.c[0 + r] * cr.w[0][k] + cr.c[3 + r] * cr.w[1][k] + cr.c[6 + r] * cr.w[2][k]) -
                     (other.c[0 + r] * other.w[0][k] + other.c[3 + r] * other.w[1][k] + other.c[6 + r] * other.w[2][k]);
      double Msch[K][K], rr[K];
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const double tk = L.total(k);
        const bool has = tk > 0.0;
        const double num = cr.num[k] + other.num[k];
        const double g = has ? num / tk - 1.0 : 0.0;
        const double Dk = has ? num / tk : 1.0;  // d g / d log, or the held identity
        const double sF = cr.s[k] + other.s[k] + wh[0][k] * XF[0] + wh[1][k] * XF[1] + wh[2][k] * XF[2];
#pragma unroll
        for (int j = 0; j < K; ++j) {
          const double SU = cr.S[k][j] + other.S[k][j] +
                            wh[0][k] * XU[0][j] + wh[1][k] * XU[1][j] + wh[2][k] * XU[2][j];
          Msch[k][j] = (j == k ? Dk : 0.0) - SU;
        }
        rr[k] = -g - sF;
      }
      small_solve<K>(Msch, rr, z);
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      double v = XF[r];
#pragma unroll
      for (int k = 0; k < K; ++k) v -= XU[r][k] * z[k];
      xm[r] = v;
    }
  }
#pragma unroll
  for (int r = 0; r < 3; ++r) xm[r] = bcast(L, xm[r]);
#pragma unroll
  for (int k = 0; k < K; ++k) z[k] = bcast(L, z[k]);

  // ---------------------------------------------------------------- back substitution
  StepOut out;
  out.size = 0.0;
  out.finite = true;
  double dlogs[K];
  if (!noise) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      dlogs[k] = clipd(z[k], -ION_LOG_CAP, ION_LOG_CAP);
      if (top) out.size = nanmax(out.size, fabs(dlogs[k]));
    }
  }
  const double QL = Q * L.L;
  const double gfrac = L.gfrac;
  CurPart cp;
  cp.zero();
  // Outward from the split: "q" is the point one position further in (new state). Half 0
  // starts with point mid + 1 as half 1 finds it (the current on interval mid is half 0's);
  // half 1 starts with none (interval mid is not its own).
  Pt pq;
  double R_q = 0.0, Ri_q[2] = {0.0, 0.0}, qv_q[2] = {0.0, 0.0}, h_q = 0.0, dx_q = 0.0;
  int ifk_q = -2;
  double U_qq[2] = {0.0, 0.0}, Ri_qq[2] = {0.0, 0.0}, b_q[2] = {0.0, 0.0};
  double Jd1[2] = {0.0, 0.0}, Jd2[2] = {0.0, 0.0};  // half 1: J of the last two inner intervals
  double A_run[2] = {0.0, 0.0}, H_run = 0.0;
  double xn[3] = {xm[0], xm[1], xm[2]};
  if (top && !noise) {
    double x1[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      double v = other.dF[r];
#pragma unroll
      for (int k = 0; k < K; ++k) v -= other.dU[r][k] * z[k];
      x1[r] = v - (other.c[r * 3 + 0] * xm[0] + other.c[r * 3 + 1] * xm[1] + other.c[r * 3 + 2] * xm[2]);
    }
    double sz_dummy = 0.0;
    bool fin_dummy = true;
    Pt px;
    px.V = xb[0]; px.lnn = xb[1]; px.lnp = xb[2];
    damp(L, x1, px, pq, sz_dummy, fin_dummy);
    pq.offn = L.st(m + 1, S_OFFN); pq.offp = L.st(m + 1, S_OFFP);
    double R, d1, d2;
    recomb(L, m + 1, pq.n, pq.p, R, d1, d2);
    const double Ug = L.st(m + 1, S_G) * gfrac;
    U_qq[0] = R - Ug; U_qq[1] = R - Ug;  // intervals mid, mid+1 hold no traps (the split's choice)
  }
  // positions nown and nown + 1 are in the ring from the forward sweep; each position stages
  // the one after it
  for (int p = nown; p >= 0; --p) {
    const int i = NODE(p);
    stage(R, p - 1, last);
    if (p > DD_PREFETCH_AHEAD) {
      prefetch_cd(L, NODE(p - DD_PREFETCH_AHEAD));
      prefetch_state(L, NODE(p - DD_PREFETCH_AHEAD));
    }
    staged_all_but_newest();  // positions p and p + 1
    Pt pi;
    if (p >= 1) {
      double x[3];
      if (p == nown && top) {
        x[0] = xm[0]; x[1] = xm[1]; x[2] = xm[2];
      } else {
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          double v = *L.cd(i, 9 + r);
          if (!noise) {
#pragma unroll
            for (int k = 0; k < K; ++k) v -= *L.cd(i, 12 + r * K + k) * z[k];
          }
          x[r] = v - (*L.cd(i, r * 3 + 0) * xn[0] + *L.cd(i, r * 3 + 1) * xn[1] + *L.cd(i, r * 3 + 2) * xn[2]);
        }
      }
      xn[0] = x[0]; xn[1] = x[1]; xn[2] = x[2];
      Pt old;
      old.V = *L.y(0, i, 0); old.lnn = *L.y(0, i, 1); old.lnp = *L.y(0, i, 2);
      if (noise) {
        const double en = exp(old.lnn), ep = exp(old.lnp);
        out.size = nanmax(out.size, fabs(x[0]) * L.iVt);
        out.size = nanmax(out.size, fabs(x[1]) * (en / (en + L.nfloor)));
        out.size = nanmax(out.size, fabs(x[2]) * (ep / (ep + L.nfloor)));
        continue;
      }
      damp(L, x, old, pi, out.size, out.finite);
      *L.y(0, i, 0) = pi.V; *L.y(0, i, 1) = pi.lnn; *L.y(0, i, 2) = pi.lnp;
    } else {
      if (noise) break;
      contact(L, top ? 0 : 1, Vint, pi);
      pi.n = exp(pi.lnn); pi.p = exp(pi.lnp);
    }
    pi.offn = R.st(i, S_OFFN); pi.offp = R.st(i, S_OFFP);
    // the interval between this point and the one further in (not half 1's at its boundary)
    const bool own_in = top || p < nown;
    const int ein = EDGE(p);
    const double h_in = R.st(ein, S_H), dx_in = R.st(ein, S_DX);
    const int ifk_in = (int)R.st(ein, S_IFK);
    double Ri_i[2] = {0.0, 0.0};
    if (own_in && ifk_in >= 0) {
      Iface t;
      if (top) iface_edge(L, ifk_in, pi.n, pq.n, pi.p, pq.p, t, false);
      else iface_edge(L, ifk_in, pq.n, pi.n, pq.p, pi.p, t, false);
      const double in_n = top ? t.v[1] : t.v[0], in_p = top ? t.v[3] : t.v[2];
      const double me_n = top ? t.v[0] : t.v[1], me_p = top ? t.v[2] : t.v[3];
      Ri_i[0] = me_n; Ri_i[1] = me_p;
      Ri_q[0] += in_n; Ri_q[1] += in_p;
    }
    double Jd[2] = {0.0, 0.0};
    if (L.currdiff && own_in) {
      const Pt& a = top ? pi : pq;
      const Pt& b = top ? pq : pi;
      Jd[0] = sg_flux(L, 0, a, b, R.st(ein, S_MUN), h_in);
      Jd[1] = sg_flux(L, 1, a, b, R.st(ein, S_MUP), h_in);
      if (ifk_in < -1) cp.dtot += h_in * (Jd[0] + Jd[1]);
    }
    // the point further in is final now: its U, the trapezoid of its inner interval, its sums
    if (p < nown) {
      const int k = NODE(p + 1);
      const double Ug = R.st(k, S_G) * gfrac;
      const double ck = 0.5 * (dx_in + dx_q);
      const bool inner_own = top || p + 1 < nown;  // half 1's boundary point: its inner interval is mid
      if (inner_own) H_run += h_q;
      const double hk = R.st(k, S_H);  // b_k takes the width of interval k
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const double sn = s == 0 ? -1.0 : 1.0;
        const double Uk = R_q + Ri_q[s] - Ug;
        if (inner_own) A_run[s] += 0.5 * dx_q * (Uk + U_qq[s]);
        cp.single[s] += ck * qv_q[s];
        cp.cq[s] += ck * qv_q[s] * A_run[s];
        const double bk = sn * QL * hk * Uk;
        cp.bH[s] += bk * H_run;
        cp.Bs[s] += bk;
        if (inner_own && ifk_q >= -1) {
          // the inner interval is a layer interface: the current through its traps, the
          // interval's physical left point's b (this point in half 0, the inner one in half 1)
          const double tk = sn * 0.5 * QL * h_q * (Ri_q[s] + Ri_qq[s]);
          cp.corr[s] += h_q * ((top ? bk : b_q[s]) - tk);
          if (L.currdiff) cp.dtot += h_q * ((top ? Jd[s] : Jd2[s]) + tk);
        }
        U_qq[s] = Uk;
        b_q[s] = bk;
      }
      Ri_qq[0] = Ri_q[0]; Ri_qq[1] = Ri_q[1];
    }
    if (!top && L.currdiff) {  // half 1 keeps the J of the intervals inside this point's
      Jd2[0] = Jd1[0]; Jd2[1] = Jd1[1];
      Jd1[0] = Jd[0]; Jd1[1] = Jd[1];
    }
    if (p >= 1) {
      double Rr, d1, d2;
      recomb(R, i, pi.n, pi.p, Rr, d1, d2);
      R_q = Rr;
    } else {
      R_q = 0.0;
    }
    qv_q[0] = DD_EXP(-(pi.V + pi.offn) * L.iVt) / R.st(i, S_MUN);
    qv_q[1] = DD_EXP((pi.V + pi.offp) * L.iVt) / R.st(i, S_MUP);
    Ri_q[0] = Ri_i[0]; Ri_q[1] = Ri_i[1];
    h_q = h_in; dx_q = dx_in; ifk_q = ifk_in;
    pq = pi;
  }
  staged_all();  // no copy into the ring left in flight (the noise step leaves the loop early)
  if (!noise) {
    // the contact: its inner interval (half 0: interval 0; half 1: interval NP, dx = 0); the
    // left contact counts in the current's sums, the right one does not (q_k for k <= NP)
    const double ck = 0.5 * dx_q;
    H_run += h_q;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      A_run[s] += 0.5 * dx_q * (0.0 + U_qq[s]);
      if (top) {
        cp.single[s] += ck * qv_q[s];
        cp.cq[s] += ck * qv_q[s] * A_run[s];
      }
      cp.A[s] = A_run[s];
    }
    cp.H = H_run;
  }
#undef NODE
#undef EDGE
  // ---------------------------------------------------------------- combine the halves
  const double osize = xchg(L, out.size);
  const int ofin = xchgi(L, out.finite ? 1 : 0);
  CurPart ot = cp;
  ot.exchange(L);
  if (top) {
    out.size = nanmax(out.size, osize);
    out.finite = out.finite && ofin;
    if (!noise) {
      const double H = L.Hsum();
      double tot = 0.0;
      if (!L.currdiff) {
        // half 0's suffix sums lack half 1's totals A_B and H_B; half 1's prefix sums are
        // subtracted from its totals
        Pt c0, cN;
        contact(L, 0, Vint, c0);
        contact(L, 1, Vint, cN);
#pragma unroll
        for (int s = 0; s < 2; ++s) {
          const double sn = s == 0 ? -1.0 : 1.0;
          const double single = cp.single[s] + ot.single[s];
          const double A = cp.A[s] + ot.A[s];
          const double cqT = cp.cq[s] + cp.single[s] * ot.A[s] + (ot.A[s] * ot.single[s] - ot.cq[s]);
          const double bH = cp.bH[s] + cp.Bs[s] * ot.H + (ot.H * ot.Bs[s] - ot.bH[s]);
          const double dbl = A * single - cqT;
          const double off0 = L.st(0, s == 0 ? S_OFFN : S_OFFP);
          const double offN = L.st(NP + 1, s == 0 ? S_OFFN : S_OFFP);
          const double d0 = exp(s == 0 ? c0.lnn : c0.lnp), dN = exp(s == 0 ? cN.lnn : cN.lnp);
          const double Kc = (L.Vt * (sn * dN * exp(sn * (cN.V + offN) * L.iVt) -
                                     sn * d0 * exp(sn * (c0.V + off0) * L.iVt)) -
                             sn * dbl) / single;
          tot += Q * Kc * H + bH - (cp.corr[s] + ot.corr[s]);
        }
      } else {
        tot = cp.dtot + ot.dtot;
      }
      out.J = -L.left() * tot / H;
    } else {
      out.J = 0.0;
    }
  }
  out.size = bcast(L, out.size);
  out.J = bcast(L, out.J);
  out.finite = bcasti(L, out.finite ? 1 : 0) != 0;
  if (!noise) {
#pragma unroll
    for (int k = 0; k < K; ++k) logs[k] += dlogs[k];
  }
  return out;
}

// ------------------------------------------------------------------------------------ start

// A point's potential and its mobile ions' densities only (the Poisson start and the ions'
// normalisations need no more of it).
template <int K>
__device__ __forceinline__ void pt_ions(const Lane& L, Pt& P, int k, const double* logs) {
  P.sl = slots_at(L, k);
  P.da = P.sl.a >= 0 ? exp(pick<K>(logs, P.sl.a) + P.V * L.iVt) : 0.0;
  P.dc = P.sl.c >= 0 ? exp(pick<K>(logs, L.ka + P.sl.c) - P.V * L.iVt) : 0.0;
}

__device__ __forceinline__ void own_range(const Lane& L, int& lo, int& hi) {
  if (L.half == 0) { lo = 1; hi = L.mid; }
  else { lo = L.mid + 1; hi = L.NP; }
}

// The normalisations that put each slot's ions into its region at the iterate's potential
// (`_ion_logs`, solver.py:1695-1725, Boltzmann ions: closed form). Each half sums its own
// intervals (half 0: 0..mid, half 1: mid+1..NP); both end with half 0's result.
template <int K>
__device__ void ion_logs(const Lane& L, double Vint, double* logs) {
  double zero[K], num[K];
#pragma unroll
  for (int k = 0; k < K; ++k) { zero[k] = 0.0; num[k] = 0.0; }
  const int m = L.mid;
  const double vb = *L.y(0, L.half == 0 ? m : m + 1, 0);
  const double vx = xchg(L, vb);
  Pt a, b;
  int e0, e1;
  if (L.half == 0) { e0 = 0; e1 = m; contact(L, 0, Vint, a); }
  else { e0 = m + 1; e1 = L.NP; a.V = vb; }
  pt_ions<K>(L, a, e0, zero);
  for (int e = e0; e <= e1; ++e) {
    if (e + 1 == L.NP + 1) contact(L, 1, Vint, b);
    else if (e + 1 == m + 1 && L.half == 0) b.V = vx;
    else b.V = *L.y(0, e + 1, 0);
    pt_ions<K>(L, b, e + 1, zero);
    ion_edge<K>(L, a, b, L.st(e, S_H) * L.L, num);
    a = b;
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const double tot = num[k] + xchg(L, num[k]);
    const double tk = L.total(k);
    logs[k] = bcast(L, tk > 0.0 ? log(tk / tot) : 0.0);
  }
}

// One Newton step of Poisson's equation alone, the densities following the potential and the
// ions re-fitted to it (`_poisson_delta`, solver.py:1757-1800; `_poisson_solve`,
// batch.py:486-503): a scalar tridiagonal system bordered by the slots, solved as the Newton
// step is (twisted, the border carried along both halves). Without mobile ions each point's step
// is clipped to 10 V_T; with them the step is scaled as a whole (its largest entry m to
// V_T ln(1 + m/V_T)). Returns max |dV| / V_T of the step taken (the same in both threads).
template <int K>
__device__ double poisson_step(Lane& L, double Vint, bool coupled, double* logs) {
  const int NP = L.NP, m = L.mid;
  const double iVt = L.iVt;
  const bool top = L.half == 0;
  ion_logs<K>(L, Vint, logs);
  bool mobile = false;
#pragma unroll
  for (int k = 0; k < K; ++k) mobile = mobile || L.total(k) > 0.0;
  mobile = mobile && coupled;
  Pt pb, px;
  const int kb = top ? m : m + 1, kx = top ? m + 1 : m;
  pb.V = *L.y(0, kb, 0); pb.lnn = *L.y(0, kb, 1); pb.lnp = *L.y(0, kb, 2);
  px.V = xchg(L, pb.V); px.lnn = xchg(L, pb.lnn); px.lnp = xchg(L, pb.lnp);
  pt_ions<K>(L, pb, kb, logs);
  pt_ions<K>(L, px, kx, logs);
  double num[K], w[K], dU[K], Sm[K][K], sv[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    num[k] = 0.0; w[k] = 0.0; dU[k] = 0.0; sv[k] = 0.0;
#pragma unroll
    for (int j = 0; j < K; ++j) Sm[k][j] = 0.0;
  }
  double c = 0.0, dF = 0.0;
  // row m (half 0 assembles it, the meeting row)
  double lo_m = 0.0, mid_m = 1.0, up_m = 0.0, F_m = 0.0, U_m[K], W_m[K];
#pragma unroll
  for (int k = 0; k < K; ++k) { U_m[k] = 0.0; W_m[k] = 0.0; }
  // one row: its coefficients and right-hand sides
  auto row = [&](int i, const Pt& pm, const Pt& pc, const Pt& pn, double hm, double hp,
                 double& lo, double& mid, double& up, double& F, double (&U)[K], double (&W)[K]) {
    const double facl = L.st(i, S_FACL), facm = L.st(i, S_FACM), facu = L.st(i, S_FACU);
    const double sP = L.st(i, S_SP);
    const double n = exp(pc.lnn), p = exp(pc.lnp);
    F = (facl * pm.V + facm * pc.V + facu * pn.V -
         Q * (n - p + L.st(i, S_DOP) + L.afix(i) + pc.da - L.cfix(i) - pc.dc)) * sP;
    mid = (facm - Q * (n + p) * iVt - Q * (pc.da + pc.dc) * iVt) * sP;
    lo = i > 1 ? facl * sP : 0.0;
    up = i < NP ? facu * sP : 0.0;
#pragma unroll
    for (int k = 0; k < K; ++k) U[k] = 0.0;
    if (pc.sl.a >= 0) set_at<K>(U, pc.sl.a, -Q * pc.da * sP);
    if (pc.sl.c >= 0) set_at<K>(U, L.ka + pc.sl.c, Q * pc.dc * sP);
    ion_w<K>(L, pm, pc, pn, hm * L.L, hp * L.L, W);
  };
  // X couples to the eliminated side, Y to the rest
  auto eliminate = [&](double X, double mid, double Y, double F, const double (&U)[K],
                       const double (&W)[K]) {
    const double im = 1.0 / (mid - X * c);
#pragma unroll
    for (int k = 0; k < K; ++k) w[k] = W[k] - c * w[k];
    dF = (-F - X * dF) * im;
#pragma unroll
    for (int k = 0; k < K; ++k) dU[k] = (U[k] - X * dU[k]) * im;
    c = Y * im;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      sv[k] += w[k] * dF;
#pragma unroll
      for (int j = 0; j < K; ++j) Sm[k][j] += w[k] * dU[j];
    }
  };
  auto store = [&](int i) {
    *L.cd(i, 0) = c;
    *L.cd(i, 1) = dF;
#pragma unroll
    for (int k = 0; k < K; ++k) *L.cd(i, 2 + k) = dU[k];
  };
  if (top) {
    Pt pm, pc, pn;
    contact(L, 0, Vint, pm);
    pt_ions<K>(L, pm, 0, logs);
    if (m == 1) pc = pb;
    else { pc.V = *L.y(0, 1, 0); pc.lnn = *L.y(0, 1, 1); pc.lnp = *L.y(0, 1, 2); pt_ions<K>(L, pc, 1, logs); }
    double h_m = L.st(0, S_H);
    ion_edge<K>(L, pm, pc, h_m * L.L, num);
    for (int i = 1; i <= m; ++i) {
      if (i + 1 == m) pn = pb;
      else if (i == m) pn = px;
      else { pn.V = *L.y(0, i + 1, 0); pn.lnn = *L.y(0, i + 1, 1); pn.lnp = *L.y(0, i + 1, 2); pt_ions<K>(L, pn, i + 1, logs); }
      const double h_i = L.st(i, S_H);
      ion_edge<K>(L, pc, pn, h_i * L.L, num);
      double lo, mid, up, F, U[K], W[K];
      row(i, pm, pc, pn, h_m, h_i, lo, mid, up, F, U, W);
      if (i < m) { eliminate(lo, mid, up, F, U, W); store(i); }
      else {
        lo_m = lo; mid_m = mid; up_m = up; F_m = F;
#pragma unroll
        for (int k = 0; k < K; ++k) { U_m[k] = U[k]; W_m[k] = W[k]; }
      }
      pm = pc; pc = pn; h_m = h_i;
    }
  } else {
    Pt pl, pc, pn;
    contact(L, 1, Vint, pn);
    pt_ions<K>(L, pn, NP + 1, logs);
    if (NP == m + 1) pc = pb;
    else { pc.V = *L.y(0, NP, 0); pc.lnn = *L.y(0, NP, 1); pc.lnp = *L.y(0, NP, 2); pt_ions<K>(L, pc, NP, logs); }
    double h_i = L.st(NP, S_H);
    ion_edge<K>(L, pc, pn, h_i * L.L, num);
    for (int i = NP; i >= m + 1; --i) {
      if (i - 1 == m) pl = px;
      else if (i - 1 == m + 1) pl = pb;
      else { pl.V = *L.y(0, i - 1, 0); pl.lnn = *L.y(0, i - 1, 1); pl.lnp = *L.y(0, i - 1, 2); pt_ions<K>(L, pl, i - 1, logs); }
      const double h_m = L.st(i - 1, S_H);
      if (i - 1 >= m + 1) ion_edge<K>(L, pl, pc, h_m * L.L, num);
      double lo, mid, up, F, U[K], W[K];
      row(i, pl, pc, pn, h_m, h_i, lo, mid, up, F, U, W);
      eliminate(up, mid, lo, F, U, W);
      store(i);
      pn = pc; pc = pl; h_i = h_m;
    }
  }
  // the meeting row
  const double c2 = xchg(L, c), dF2 = xchg(L, dF);
  double dU2[K], w2[K], S2[K][K], s2[K], num2[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    dU2[k] = xchg(L, dU[k]); w2[k] = xchg(L, w[k]); s2[k] = xchg(L, sv[k]); num2[k] = xchg(L, num[k]);
#pragma unroll
    for (int j = 0; j < K; ++j) S2[k][j] = xchg(L, Sm[k][j]);
  }
  double z[K], xm = 0.0;
#pragma unroll
  for (int k = 0; k < K; ++k) z[k] = 0.0;
  if (top) {
    const double ig = 1.0 / (mid_m - lo_m * c - up_m * c2);
    const double XF = (-F_m - lo_m * dF - up_m * dF2) * ig;
    double XU[K];
#pragma unroll
    for (int k = 0; k < K; ++k) XU[k] = (U_m[k] - lo_m * dU[k] - up_m * dU2[k]) * ig;
    if (mobile) {
      double Msch[K][K], rr[K];
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const double wh = W_m[k] - c * w[k] - c2 * w2[k];
        const double tk = L.total(k);
        const bool has = tk > 0.0;
        const double nm = num[k] + num2[k];
        const double g = has ? nm / tk - 1.0 : 0.0;
        const double Dk = has ? nm / tk : 1.0;
#pragma unroll
        for (int j = 0; j < K; ++j) Msch[k][j] = (j == k ? Dk : 0.0) - (Sm[k][j] + S2[k][j] + wh * XU[j]);
        rr[k] = -g - (sv[k] + s2[k] + wh * XF);
      }
      small_solve<K>(Msch, rr, z);
    }
    xm = XF;
#pragma unroll
    for (int k = 0; k < K; ++k) xm -= XU[k] * z[k];
  }
  xm = bcast(L, xm);
#pragma unroll
  for (int k = 0; k < K; ++k) z[k] = bcast(L, z[k]);
  const double capV = CAP_V * L.Vt;
  double mx = 0.0, size = 0.0;
  auto apply = [&](int i, double dV) {
    *L.y(0, i, 0) += dV;
    *L.y(0, i, 1) += dV * iVt;
    *L.y(0, i, 2) -= dV * iVt;
    size = nanmax(size, fabs(dV * iVt));
  };
  auto visit = [&](int i, double x) {
    if (mobile) {
      *L.cd(i, 1) = x;
      mx = nanmax(mx, fabs(x) * iVt);
    } else {
      apply(i, clipd(x, -capV, capV));
    }
  };
  if (top) {
    double x = xm;
    visit(m, x);
    for (int i = m - 1; i >= 1; --i) {
      double v = *L.cd(i, 1);
#pragma unroll
      for (int k = 0; k < K; ++k) v -= *L.cd(i, 2 + k) * z[k];
      x = v - *L.cd(i, 0) * x;
      visit(i, x);
    }
  } else {
    double x = xm;
    for (int i = m + 1; i <= NP; ++i) {
      double v = *L.cd(i, 1);
#pragma unroll
      for (int k = 0; k < K; ++k) v -= *L.cd(i, 2 + k) * z[k];
      x = v - *L.cd(i, 0) * x;
      visit(i, x);
    }
  }
  if (mobile) {
    mx = nanmax(mx, xchg(L, mx));
    mx = bcast(L, mx);
    const double f = mx > 0.0 ? fmin(log1p(mx), CAP_V) / mx : 1.0;
    int lo, hi;
    own_range(L, lo, hi);
    for (int i = lo; i <= hi; ++i) apply(i, *L.cd(i, 1) * f);
  }
  size = nanmax(size, xchg(L, size));
  return bcast(L, size);
}

// The mobile ions of the iterate as fixed densities, no longer solved for (`_freeze`,
// batch.py:859-872). Each half its own points.
template <int K>
__device__ void freeze(Lane& L, const double* logs) {
  int lo, hi;
  own_range(L, lo, hi);
  for (int i = lo; i <= hi; ++i) {
    Pt P;
    P.V = *L.y(0, i, 0);
    pt_ions<K>(L, P, i, logs);
    L.FX[((size_t)i * 2) * L.Bp + L.l] = L.afix(i) + P.da;
    L.FX[((size_t)i * 2 + 1) * L.Bp + L.l] = L.cfix(i) + P.dc;
  }
  L.frozen = true;
}

// The iterate (each half its own points) and the normalisations (half 0) into a checkpoint.
template <int K>
__device__ void save_state(const Lane& L, double* ys, double* ls, const double* logs) {
  int lo, hi;
  own_range(L, lo, hi);
  for (int i = lo; i <= hi; ++i)
#pragma unroll
    for (int c = 0; c < 3; ++c) ys[((size_t)i * 3 + c) * L.Bp + L.l] = *L.y(0, i, c);
  if (L.half == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) ls[(size_t)k * L.Bp + L.l] = logs[k];
}

__device__ void copy_state(const Lane& L, int dst, int src) {
  int lo, hi;
  own_range(L, lo, hi);
  for (int i = lo; i <= hi; ++i)
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
  // dd_solve_states: the converged states per voltage (null for dd_solve)
  double* states;        // [nv_max][np+2][3][Bp]
  double* state_logs;    // [nv_max][DD_MAXK][Bp]
  double* prebias;       // [np+2][3][Bp]
  double* prebias_logs;  // [DD_MAXK][Bp]
  int nv_max;
  // the work queue (null: one device per pair): its counter and the pairs of the grid
  int* queue;
  int pairs;
  // 1: only the lanes with the differential current (the generic kernel's second launch after
  // the specialised one, which leaves them)
  int diff_only;
  // dd_newton_step
  double* logs_io;
  const double* vint;
  double share;
  double* size_out;
  double* J_out;
};

template <int K>
__device__ void lane_init(Lane& L, const Args& a, int l, int half) {
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
  L.Y = a.Y; L.FX = a.FX; L.CD = a.CD; L.ncd = a.ncd;
  L.ybuf = (size_t)(a.npmax + 2) * 3 * a.Bp;
  L.frozen = false;
  L.share = 1.0;
  L.half = half;
  const int wl = threadIdx.x & 31;
  L.base = wl & ~1;
  L.mask = 3u << L.base;
}

// One lane's program bookkeeping between Newton steps (see solve_kernel).
template <int K>
struct Prog {
  double lgA[K], lgB[K], lgC[K];  // normalisations: last carry, the one before, the stage start
  double hs[4], hJ[4];            // the last four steps' sizes and currents
  double noise_floor, before, Vlast, Vbefore;
  int pit, ctx, it, cap, nsz, stage, k, below, last_keep, jcur, n_border, n_plain;
  bool floor_known, pending_noise, ok_f, kept_f, solved, pre_ok, ok_c;
};

enum Phase { PH_POISSON = 0, PH_NEWTON, PH_DONE };
enum Ctx {
  X_START_F = 0, X_STAGE, X_PRE, X_SCAN,          // solve_batch (batch.py:875-1006)
  X_JV_START, X_JV_STAGE, X_JV_PRE, X_JV_SCAN     // solve_jv (solver.py:2105-2245)
};

// The whole J-V program of one device, run by both threads of its pair: every decision is
// taken on values both hold bit for bit (half 0's, broadcast), so the two never part ways.
template <int K, int BS, bool GENERIC>
__device__ __forceinline__ void run_lane(const Args& a, int l, int half, Prog<K>& g,
                                         double* ring) {
  Lane L;
  lane_init<K>(L, a, l, half);
  // The common launch (batch mode, the exact Bernoulli function, the integral current) is
  // compiled without the others' paths, which would otherwise sit in the sweeps' code and cost
  // instruction fetch: it leaves the lanes with the differential current to a second launch of
  // the generic kernel, which takes those alone.
  if (!GENERIC) {
    L.simss = 0;
    if (L.currdiff) return;
    L.currdiff = 0;
  } else if (a.diff_only && !L.currdiff) {
    return;
  }
  const bool top = half == 0;
  const bool jv = GENERIC && a.mode == DD_MODE_JV;
  const int voff = a.voff[l], nv = a.vcnt[l];
  if (nv <= 0) return;
  const double* Vl = a.V + voff;
  const bool pre_cond = L.sc(C_PRECOND) > 0.0, fix_ions = L.sc(C_FIXIONS) > 0.0;
  const double first = pre_cond ? L.sc(C_VPRE) : Vl[0];
  {
    int lo, hi;
    own_range(L, lo, hi);
    for (int i = lo; i <= hi; ++i)
#pragma unroll
      for (int c = 0; c < 3; ++c) *L.y(0, i, c) = __ldg(a.Y0 + ((size_t)i * 3 + c) * a.Bp + l);
  }
  bool mobile = false;
#pragma unroll
  for (int q = 0; q < K; ++q) mobile = mobile || L.tot[q] > 0.0;

  double logs[K];
#pragma unroll
  for (int q = 0; q < K; ++q) { logs[q] = 0.0; g.lgA[q] = 0.0; g.lgB[q] = 0.0; g.lgC[q] = 0.0; }
  int phase = PH_POISSON;
  g.pit = 0;
  const int pcap = jv ? a.max_iter : a.start_iter;
  int adv = ADV_NONE;
  g.ctx = 0; g.it = 0; g.cap = 0;
  double Vint = first, ratio = 0.0;
  g.nsz = 0;
  g.floor_known = false; g.pending_noise = false;
  g.noise_floor = 0.0;
  g.ok_f = false; g.kept_f = false; g.solved = false; g.pre_ok = true; g.ok_c = false;
  g.stage = 0;
  g.before = 1.0;
  g.k = 0; g.below = 0; g.last_keep = 0;
  g.Vlast = first; g.Vbefore = first;
  g.jcur = 0;
  g.n_border = 0; g.n_plain = 0;
  if (!jv) {
    while (g.below < nv && Vl[g.below] < first) ++g.below;  // searchsorted, left
  }
  if (top) a.status[l] = DD_LANE_OK;

  auto begin = [&](int c, double v, double share, int cp_, int ad, double ra) {
    g.ctx = c; Vint = v; L.share = share; g.cap = cp_; adv = ad; ratio = ra;
    g.it = 0; g.nsz = 0; g.floor_known = false; g.pending_noise = false;
#pragma unroll
    for (int q = 0; q < 4; ++q) { g.hs[q] = INFINITY; g.hJ[q] = INFINITY; }
    phase = PH_NEWTON;
  };
  auto scan_begin = [&]() {
    if (g.k >= nv) { phase = PH_DONE; return; }
    if (!jv) {
      g.jcur = g.k < nv - g.below ? g.below + g.k : nv - 1 - g.k;
      const double v = Vl[g.jcur];
      if (g.k == 0 || g.k == nv - g.below) {
        g.Vlast = first; g.Vbefore = first;
        copyv<K>(logs, g.lgC); copyv<K>(g.lgA, g.lgC); copyv<K>(g.lgB, g.lgC);
        begin(X_SCAN, v, 1.0, a.max_iter, ADV_TURN, 0.0);
      } else {
        const double ra = g.Vlast != g.Vbefore ? (v - g.Vlast) / (g.Vlast - g.Vbefore) : 0.0;
#pragma unroll
        for (int q = 0; q < K; ++q)
          logs[q] = g.lgA[q] + (ra != 0.0 ? clipd(ra * (g.lgA[q] - g.lgB[q]), -ION_LOG_CAP, ION_LOG_CAP) : 0.0);
        begin(X_SCAN, v, 1.0, a.max_iter, g.last_keep ? ADV_KEEP : ADV_NOKEEP, ra);
      }
    } else {
      g.jcur = g.k;
      copyv<K>(logs, g.lgA);
      begin(X_JV_SCAN, Vl[g.k], 1.0, a.max_iter, g.last_keep ? ADV_KEEP : ADV_NOKEEP, 0.0);
    }
  };
  auto freeze_and_scan = [&]() {
    L.share = 1.0;
    if (a.prebias) save_state<K>(L, a.prebias, a.prebias_logs, logs);
    if (!jv) {
      const bool fr = pre_cond && fix_ions;
      if (fr) freeze<K>(L, logs);
      g.pre_ok = g.pre_ok || !fr;
      copy_state(L, 3, 0);
      copyv<K>(g.lgC, logs);
      g.k = 0;
      scan_begin();
    } else {
      if (pre_cond && fix_ions) freeze<K>(L, logs);
      copy_state(L, 1, 0);  // the carry: the first voltage's ADV_KEEP reads it
      copyv<K>(g.lgA, logs);
      g.k = 0; g.last_keep = 1;  // the start is the carry
      scan_begin();
    }
  };
  auto batch_pre = [&]() {
    L.share = 1.0;
    if (g.solved) { g.pre_ok = true; freeze_and_scan(); }
    else begin(X_PRE, first, 1.0, a.start_iter, ADV_NONE, 0.0);
  };
  auto stage_begin = [&]() {
    const double share = c_stage_share[g.stage];
    const double sh = log(share / g.before);
#pragma unroll
    for (int q = 0; q < K; ++q) logs[q] += sh;
    if (!jv) { copy_state(L, 3, 0); copyv<K>(g.lgC, logs); }
    begin(jv ? X_JV_STAGE : X_STAGE, first, share, jv ? a.max_iter : a.start_iter, ADV_NONE, 0.0);
  };
  auto jv_pre = [&]() {
    L.share = 1.0;
    if (pre_cond) begin(X_JV_PRE, L.sc(C_VPRE), 1.0, a.max_iter, ADV_NONE, 0.0);
    else freeze_and_scan();
  };

  while (phase != PH_DONE) {
    if (phase == PH_POISSON) {
      const double size = poisson_step<K>(L, first, jv ? mobile : true, logs);
      ++g.pit;
      const bool stop = jv ? (size < POISSON_TOL || g.pit >= pcap) : (!(size > POISSON_TOL) || g.pit >= pcap);
      if (!stop) continue;
      ion_logs<K>(L, first, logs);
      if (!jv) {
        copy_state(L, 1, 0);
        copyv<K>(g.lgA, logs);
        begin(X_START_F, first, 1.0, a.start_iter, ADV_NONE, 0.0);
      } else if (mobile) {
        copy_state(L, 1, 0);
        copyv<K>(g.lgA, logs);
        begin(X_JV_START, first, 1.0, a.max_iter, ADV_NONE, 0.0);
      } else {
        jv_pre();
      }
      continue;
    }
    bool end = false, conv = false, fin = true;
    double Jv = 0.0;
    // one call site of the step (the round-off step with `noise`): the step's code once
    const bool noise = GENERIC && g.pending_noise;
    const StepOut o = newton_step<K, BS>(L, Vint, logs, noise ? (int)ADV_NONE : adv,
                                     noise ? 0.0 : ratio, noise, ring);
    if (noise) {
      ++g.n_plain;
      g.noise_floor = o.size; g.floor_known = true; g.pending_noise = false;
      double mx = 0.0;
      for (int q = 4 - (g.nsz < 4 ? g.nsz : 4); q < 4; ++q) mx = nanmax(mx, g.hs[q]);
      if (mx < g.noise_floor) { end = true; conv = true; }
      else if (g.it >= g.cap) { end = true; conv = false; }
      Jv = g.hJ[3];
      if (!end) continue;
    } else {
      adv = ADV_NONE;
      ++g.it;
      bool border = false;
#pragma unroll
      for (int q = 0; q < K; ++q) border = border || L.total(q) > 0.0;
      if (border) ++g.n_border; else ++g.n_plain;
#pragma unroll
      for (int q = 0; q < 3; ++q) { g.hs[q] = g.hs[q + 1]; g.hJ[q] = g.hJ[q + 1]; }
      g.hs[3] = o.size; g.hJ[3] = o.J;
      ++g.nsz;
      Jv = o.J;
      fin = o.finite && finitev<K>(logs);
      const double size = o.size;
      const bool isn = size != size;
      const bool settle = g.ctx >= X_JV_START;
      if (!settle) {
        double mx = g.hs[0], mn = g.hs[1];
#pragma unroll
        for (int q = 1; q < 4; ++q) mx = nanmax(mx, g.hs[q]);
#pragma unroll
        for (int q = 2; q < 4; ++q) mn = (g.hs[q] < mn || g.hs[q] != g.hs[q]) ? g.hs[q] : mn;
        const bool stalled = g.it > STALL_STEPS && mx < ROUND_OFF_FLOOR && mn >= 0.1 * g.hs[0];
        double dJ = 0.0;
#pragma unroll
        for (int q = 0; q < 4; ++q) dJ = nanmax(dJ, fabs(g.hJ[q] - g.hJ[3]));
        const bool settled = g.it > STALL_STEPS && size < CURRENT_STEP_CAP &&
                             dJ < CURRENT_TOL * (L.Jscale() + fabs(g.hJ[3]));
        const bool quad = g.it > 1 && size < QUADRATIC_TOL && size < QUADRATIC_RATIO * g.hs[2];
        conv = a.strict ? (size < a.tol || stalled) : (size < a.tol || stalled || settled || quad);
        end = conv || g.it >= g.cap || isn;
      } else {
        if (isn) { end = true; conv = false; }
        else {
          const int n4 = g.nsz < 4 ? g.nsz : 4;
          double mx = 0.0, mn = INFINITY;
          for (int q = 4 - n4; q < 4; ++q) mx = nanmax(mx, g.hs[q]);
          for (int q = 4 - n4 + 1; q < 4; ++q) mn = fmin(mn, g.hs[q]);
          bool done = size < a.tol || (g.nsz >= 4 && mx < ROUND_OFF_FLOOR && mn >= 0.1 * g.hs[0]);
          if (!done && g.nsz >= 4 && mx < NOISE_FLOOR_CAP) {
            if (!g.floor_known) { g.pending_noise = true; continue; }
            done = mx < g.noise_floor;
          }
          if (done) { end = true; conv = true; }
          else if (g.it >= g.cap) { end = true; conv = false; }
        }
      }
      if (!end) continue;
    }
    switch (g.ctx) {
      case X_START_F: {
        g.ok_f = conv; g.kept_f = fin;
        if (g.ok_f || !mobile) {
          if (!g.kept_f) { copy_state(L, 0, 1); copyv<K>(logs, g.lgA); }
          g.solved = g.ok_f;
          batch_pre();
        } else {
          copy_state(L, 2, 0); copyv<K>(g.lgB, logs);
          copy_state(L, 0, 1); copyv<K>(logs, g.lgA);
          g.before = 1.0; g.stage = 0;
          stage_begin();
        }
        break;
      }
      case X_STAGE: {
        g.ok_c = conv;
        if (!fin) { copy_state(L, 0, 3); copyv<K>(logs, g.lgC); }
        g.before = c_stage_share[g.stage];
        ++g.stage;
        if (g.stage < 4) { stage_begin(); break; }
        const bool staged = g.ok_c;
        if (!staged) {
          if (g.kept_f) { copy_state(L, 0, 2); copyv<K>(logs, g.lgB); }
          else { copy_state(L, 0, 1); copyv<K>(logs, g.lgA); }
        }
        g.solved = staged;
        batch_pre();
        break;
      }
      case X_PRE: {
        g.pre_ok = conv;
        freeze_and_scan();
        break;
      }
      case X_SCAN: {
        const int pos = voff + g.jcur;
        if (top) {
          a.J[pos] = Jv + L.Gshunt() * Vint;
          a.ok[pos] = (conv && g.pre_ok) ? 1 : 0;
          a.its[pos] = g.it;
        }
        if (a.states && g.jcur < a.nv_max)
          save_state<K>(L, a.states + (size_t)g.jcur * (a.npmax + 2) * 3 * a.Bp,
                        a.state_logs + (size_t)g.jcur * DD_MAXK * a.Bp, logs);
        const bool keep = conv && fin;
        if (keep) {
          copyv<K>(g.lgB, g.lgA); copyv<K>(g.lgA, logs);
          g.Vbefore = g.Vlast; g.Vlast = Vint; g.last_keep = 1;
        } else {
          g.last_keep = 0;
        }
        ++g.k;
        scan_begin();
        break;
      }
      case X_JV_START: {
        if (conv) { jv_pre(); break; }
        copy_state(L, 0, 1); copyv<K>(logs, g.lgA);
        g.before = 1.0; g.stage = 0;
        stage_begin();
        break;
      }
      case X_JV_STAGE: {
        g.before = c_stage_share[g.stage];
        if (!conv) { copy_state(L, 0, 1); copyv<K>(logs, g.lgA); jv_pre(); break; }
        ++g.stage;
        if (g.stage < 4) stage_begin();
        else jv_pre();
        break;
      }
      case X_JV_PRE: {
        if (!conv) {
          if (top) {
            a.status[l] = DD_LANE_PREBIAS_FAILED;
            for (int q = 0; q < nv; ++q) { a.J[voff + q] = NAN; a.ok[voff + q] = 0; a.its[voff + q] = 0; }
          }
          phase = PH_DONE;
          break;
        }
        freeze_and_scan();
        break;
      }
      case X_JV_SCAN: {
        const int pos = voff + g.jcur;
        if (top) {
          a.J[pos] = Jv + L.Gshunt() * Vint;
          a.ok[pos] = conv ? 1 : 0;
          a.its[pos] = g.it;
        }
        if (a.states && g.jcur < a.nv_max)
          save_state<K>(L, a.states + (size_t)g.jcur * (a.npmax + 2) * 3 * a.Bp,
                        a.state_logs + (size_t)g.jcur * DD_MAXK * a.Bp, logs);
        const bool keep = conv && fin;
        if (keep) { copyv<K>(g.lgA, logs); g.last_keep = 1; }
        else g.last_keep = 0;
        ++g.k;
        scan_begin();
        break;
      }
    }
  }
  if (a.steps && top) {
    a.steps[l] = g.n_border;
    a.steps[a.Bp + l] = g.n_plain;
    a.steps[2 * a.Bp + l] = g.pit;
  }
}

// The solve: each pair of threads runs one device's whole program (run_lane). With a work queue
// (`a.queue`, a batch of more devices than the GPU holds at once) the grid is what the GPU holds
// and a pair that finishes a device takes the next one from the queue, so no pair waits for the
// slowest device of its warp; devices are taken in lane order (the packer puts the largest
// grids first). The program's bookkeeping between steps lives in shared memory (one record per
// thread), so that the sweeps have the registers to themselves, beside the sweeps' ring. BS
// threads a block; the ring (RING * DD_NF * BS words) is the launch's dynamic shared memory.
// GENERIC: any mode and Bernoulli function; otherwise batch mode with the exact one only.
template <int K, int BS, bool GENERIC>
__global__ void __launch_bounds__(64) solve_kernel(Args a) {
  __shared__ Prog<K> progs[BS];
  extern __shared__ double ring[];
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int half = tid & 1;
  const int base = (threadIdx.x & 31) & ~1;
  const unsigned pair = 3u << base;
  int l = tid >> 1;
  while (l < a.B) {
    run_lane<K, BS, GENERIC>(a, l, half, progs[threadIdx.x], ring + threadIdx.x);
    if (!a.queue) break;
    int next = 0;
    if (half == 0) next = a.pairs + atomicAdd(a.queue, 1);
    l = __shfl_sync(pair, next, base);
  }
}

// One Newton step per lane from a given state (dd_newton_step).
template <int K>
__global__ void __launch_bounds__(64) step_kernel(Args a) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int l = tid >> 1, half = tid & 1;
  if (l >= a.B) return;
  Lane L;
  lane_init<K>(L, a, l, half);
  L.share = a.share;
  double logs[K];
#pragma unroll
  for (int k = 0; k < K; ++k) logs[k] = a.logs_io[(size_t)k * a.Bp + l];
  __shared__ double ring[RING * DD_NF * DD_SOLVE_BLOCK];
  const StepOut o = newton_step<K, DD_SOLVE_BLOCK>(L, a.vint[l], logs, ADV_NONE, 0.0, false,
                                                   ring + threadIdx.x);
  if (half == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) a.logs_io[(size_t)k * a.Bp + l] = logs[k];
    a.size_out[l] = o.size;
    a.J_out[l] = o.J;
  }
}

}  // namespace dd

// ======================================================================================== C ABI

namespace {

int slots_k(const dd_batch* b) { return b->k_anion + b->k_cation <= 2 ? 2 : 4; }


// The work queue's counter: its own 256 bytes at the workspace's end.
constexpr size_t QUEUE_ELEMS = 32;

size_t ws_elems(const dd_batch* b, size_t* y_e, size_t* fx_e, size_t* cd_e, int* ncd) {
  const int K = slots_k(b);
  *ncd = 12 + 3 * K;
  const size_t nodes = (size_t)b->np_max + 2;
  *y_e = (size_t)dd::DD_NBUF * nodes * 3 * b->lane_stride;
  *fx_e = nodes * 2 * b->lane_stride;
  *cd_e = nodes * (size_t)(*ncd) * b->lane_stride;
  return *y_e + *fx_e + *cd_e + QUEUE_ELEMS;
}

// ------------------------------------------------------------------ launch forms and tuning
//
// A launch form of the solve: threads per block (two per device) and whether a batch of more
// devices than the GPU holds at once runs from the work queue (as many pairs as the GPU holds,
// each taking the next device when done) or as one pair per device (the hardware starting
// blocks as others finish). Every form gives the same results. `dd_tune` times them on a batch
// and keeps the fastest for batches of its shape; untuned shapes take form 0.
struct Form {
  int block;
  bool queue;
};
constexpr Form FORMS[DD_SOLVE_FORMS] = {{32, true}, {64, true}, {32, false}, {64, false}};

template <int K>
const void* solve_kernel_ptr(int block, bool generic) {
  if (generic)
    return block == 64 ? (const void*)dd::solve_kernel<K, 64, true>
                       : (const void*)dd::solve_kernel<K, 32, true>;
  return block == 64 ? (const void*)dd::solve_kernel<K, 64, false>
                     : (const void*)dd::solve_kernel<K, 32, false>;
}

// The dynamic shared memory of a block (the sweeps' ring), allowed above the default 48 KB a
// block for the 64-thread form.
size_t ring_bytes(int block) { return sizeof(double) * dd::RING * dd::DD_NF * block; }

bool allow_ring(const void* kernel, int block) {
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)ring_bytes(block)) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return true;
}

// The pairs the GPU holds at once for this kernel and block size (its occupancy), 0 if unknown.
long pairs_held(const void* kernel, int block) {
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, ring_bytes(block)) !=
          cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return (long)sms * per_sm * (block / 2);
}

// Launch the solve in form `f`: the work queue's counter (the workspace's last 256 bytes) is
// zeroed on the stream first when the queue is used.
int launch_solve(const dd_batch* b, dd::Args& a, void* ws, cudaStream_t s, const Form& f) {
  const int K = slots_k(b);
  auto go = [&](bool generic) {
    const void* kernel = K == 2 ? solve_kernel_ptr<2>(f.block, generic)
                                : solve_kernel_ptr<4>(f.block, generic);
    if (!allow_ring(kernel, f.block)) return DD_ERR_LAUNCH;
    const long held = f.queue ? pairs_held(kernel, f.block) : 0;
    a.queue = nullptr;
    a.pairs = 0;
    dim3 grid((2 * b->lane_stride + f.block - 1) / f.block);
    if (held > 0 && b->n_lanes > held) {
      size_t ye, fe, ce;
      int ncd;
      const size_t at = ws_elems(b, &ye, &fe, &ce, &ncd) - QUEUE_ELEMS;
      a.queue = reinterpret_cast<int*>(static_cast<double*>(ws) + at);
      a.pairs = (int)held;
      if (cudaMemsetAsync(a.queue, 0, sizeof(int), s) != cudaSuccess) return DD_ERR_LAUNCH;
      grid = dim3((unsigned)(2 * held / f.block));
    }
    void* args[] = {&a};
    return cudaLaunchKernel(kernel, grid, dim3(f.block), args, ring_bytes(f.block), s) ==
                   cudaSuccess
               ? DD_OK
               : DD_ERR_LAUNCH;
  };
  // batch mode with the exact Bernoulli function: the specialised kernel, then the generic one
  // for the lanes with the differential current (it returns at once for the others); else the
  // generic one alone
  a.diff_only = 0;
  if (a.mode != DD_MODE_BATCH || a.simss) return go(true);
  const int st = go(false);
  if (st != DD_OK) return st;
  a.diff_only = 1;
  const int st2 = go(true);
  a.diff_only = 0;
  return st2;
}

// The tuned forms of this process: by device, ion slots, grid size and lane count (within a
// factor of two).
struct TuneKey {
  int dev, K, np_max, lanes_log2;
  bool operator==(const TuneKey& o) const {
    return dev == o.dev && K == o.K && np_max == o.np_max && lanes_log2 == o.lanes_log2;
  }
};
std::mutex tune_mutex;
std::vector<std::pair<TuneKey, int>> tuned;

bool tune_key(const dd_batch* b, TuneKey& k) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  int lg = 0;
  while ((1L << lg) < b->n_lanes) ++lg;
  k = TuneKey{dev, slots_k(b), b->np_max, lg};
  return true;
}

const Form& form_for(const dd_batch* b) {
  TuneKey k;
  if (tune_key(b, k)) {
    std::lock_guard<std::mutex> guard(tune_mutex);
    for (const auto& e : tuned)
      if (e.first == k) return FORMS[e.second];
  }
  return FORMS[0];
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
    case DD_ERR_SCRATCH: return "batch needs more scratch than dd_solve_noalloc's fixed array";
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
  if ((st = dd::device_status()) != DD_OK) return st;
  dd::Args a = make_args(batch, workspace);
  a.V = volts->v; a.voff = volts->offset; a.vcnt = volts->count;
  a.J = J; a.ok = converged; a.its = iterations; a.status = lane_status; a.steps = lane_steps;
  a.tol = opts->tol; a.max_iter = opts->max_iter; a.start_iter = opts->start_iter;
  a.strict = opts->strict; a.simss = opts->bernoulli == DD_BERNOULLI_SIMSS; a.mode = opts->mode;
  return launch_solve(batch, a, workspace, static_cast<cudaStream_t>(stream), form_for(batch));
}

int dd_solve_states(const dd_batch* batch, const dd_voltages* volts, const dd_opts* opts,
                    double* J, uint8_t* converged, int32_t* iterations, int32_t* lane_status,
                    int32_t* lane_steps, double* states, double* state_logs, double* prebias,
                    double* prebias_logs, int nv_max, void* workspace, size_t workspace_bytes,
                    void* stream) {
  int st = check_batch(batch);
  if (st != DD_OK) return st;
  if (!volts || !volts->v || !volts->offset || !volts->count || !opts || !J || !converged ||
      !iterations || !lane_status || !workspace || !states || !state_logs || !prebias ||
      !prebias_logs || nv_max < 1)
    return DD_ERR_ARGS;
  if (opts->max_iter < 1 || opts->start_iter < 1 || (opts->mode != DD_MODE_BATCH && opts->mode != DD_MODE_JV) ||
      (opts->bernoulli != DD_BERNOULLI_EXACT && opts->bernoulli != DD_BERNOULLI_SIMSS) ||
      opts->precision != DD_PRECISION_FP64)
    return DD_ERR_ARGS;
  size_t need;
  dd_workspace_bytes(batch, &need);
  if (workspace_bytes < need) return DD_ERR_WORKSPACE;
  if ((st = dd::device_status()) != DD_OK) return st;
  dd::Args a = make_args(batch, workspace);
  a.V = volts->v; a.voff = volts->offset; a.vcnt = volts->count;
  a.J = J; a.ok = converged; a.its = iterations; a.status = lane_status; a.steps = lane_steps;
  a.tol = opts->tol; a.max_iter = opts->max_iter; a.start_iter = opts->start_iter;
  a.strict = opts->strict; a.simss = opts->bernoulli == DD_BERNOULLI_SIMSS; a.mode = opts->mode;
  a.states = states; a.state_logs = state_logs; a.prebias = prebias;
  a.prebias_logs = prebias_logs; a.nv_max = nv_max;
  return launch_solve(batch, a, workspace, static_cast<cudaStream_t>(stream), form_for(batch));
}

int dd_tune(const dd_batch* batch, const dd_voltages* volts, const dd_opts* opts, double* J,
            uint8_t* converged, int32_t* iterations, int32_t* lane_status, int32_t* lane_steps,
            void* workspace, size_t workspace_bytes, void* stream, int32_t* form,
            float* times_ms) {
  if (!form) return DD_ERR_ARGS;
  int st = check_batch(batch);
  if (st != DD_OK) return st;
  TuneKey key;
  if (!tune_key(batch, key)) return DD_ERR_DEVICE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) {
    cudaGetLastError();
    return DD_ERR_LAUNCH;
  }
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaGetLastError();
    cudaEventDestroy(e0);
    return DD_ERR_LAUNCH;
  }
  int best = -1;
  float best_ms = 0.0f;
  for (int f = 0; f < DD_SOLVE_FORMS && st == DD_OK; ++f) {
    {  // the form being timed is the shape's form for this one solve
      std::lock_guard<std::mutex> guard(tune_mutex);
      bool found = false;
      for (auto& e : tuned)
        if (e.first == key) { e.second = f; found = true; }
      if (!found) tuned.push_back({key, f});
    }
    float ms = 0.0f;
    if (cudaEventRecord(e0, s) != cudaSuccess) st = DD_ERR_LAUNCH;
    if (st == DD_OK)
      st = dd_solve(batch, volts, opts, J, converged, iterations, lane_status, lane_steps,
                    workspace, workspace_bytes, stream);
    if (st == DD_OK && (cudaEventRecord(e1, s) != cudaSuccess ||
                        cudaEventSynchronize(e1) != cudaSuccess ||
                        cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
      st = DD_ERR_LAUNCH;
    if (st == DD_OK) {
      if (times_ms) times_ms[f] = ms;
      if (best < 0 || ms < best_ms) { best = f; best_ms = ms; }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  {
    std::lock_guard<std::mutex> guard(tune_mutex);
    for (auto& e : tuned)
      if (e.first == key) e.second = best < 0 ? 0 : best;
  }
  if (st != DD_OK) return st;
  *form = best;
  return DD_OK;
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
  if ((st = dd::device_status()) != DD_OK) return st;
  dd::Args a = make_args(batch, workspace);
  a.Y = y;  // the caller's state is the iterate buffer
  a.simss = opts->bernoulli == DD_BERNOULLI_SIMSS;
  a.logs_io = logs; a.vint = vint; a.share = share; a.size_out = size; a.J_out = J;
  const dim3 grid((2 * batch->lane_stride + DD_SOLVE_BLOCK - 1) / DD_SOLVE_BLOCK),
      block(DD_SOLVE_BLOCK);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  return slots_k(batch) == 2 ? dd::launch(dd::step_kernel<2>, grid, block, 0, s, a)
                             : dd::launch(dd::step_kernel<4>, grid, block, 0, s, a);
}

}  // extern "C"

// ===================================================== allocation-free solve (dd_solve_noalloc)
//
// The scratch lives in one fixed array in the library's own device memory, reserved when the
// module loads on a device. Every call on a device uses the same array: whatever the last call
// left there stays, and two calls whose launches overlap (two streams, two host threads) race on
// it. The solve kernel writes each word of its scratch before it reads it (the starting state
// from y0, the sweep's records node by node, the carries before any voltage's start reads them),
// so nothing has to be cleared between calls.

namespace {

static __device__ __align__(256) double noalloc_scratch[DD_NOALLOC_SCRATCH_BYTES / sizeof(double)];

constexpr int kMaxDevices = 64;
std::mutex noalloc_mutex;
// per device: the array's address and the id of the context it was looked up in
void* noalloc_ptr[kMaxDevices] = {};
unsigned long long noalloc_ctx[kMaxDevices] = {};

// The driver's id of the context current on this thread (0 when there is none, or the driver
// does not offer the query). A context torn down and re-created (cudaDeviceReset, then any
// runtime call) gets a new id, and the library's module, with this array, is loaded anew in it.
unsigned long long current_context_id() {
  using GetCurrent = int (*)(void**);
  using GetId = int (*)(void*, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault) == cudaSuccess && f)
      get_current = reinterpret_cast<GetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault) == cudaSuccess && f)
      get_id = reinterpret_cast<GetId>(f);
    cudaGetLastError();  // a failed lookup is not the caller's error
  });
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

// The array's address on the current device, looked up (with that device current) on the first
// call and again whenever the device's context is not the one of the last lookup; nullptr if
// there is no usable device or the lookup failed.
void* noalloc_scratch_ptr() {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return nullptr;
  }
  std::lock_guard<std::mutex> guard(noalloc_mutex);
  const unsigned long long ctx = current_context_id();
  if (!noalloc_ptr[dev] || ctx == 0 || ctx != noalloc_ctx[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, noalloc_scratch) != cudaSuccess || !p) {
      cudaGetLastError();  // so that the caller's next cudaGetLastError does not report it
      noalloc_ptr[dev] = nullptr;
      return nullptr;
    }
    noalloc_ptr[dev] = p;
    // the lookup made the device's primary context current if none was
    noalloc_ctx[dev] = ctx != 0 ? ctx : current_context_id();
  }
  return noalloc_ptr[dev];
}

}  // namespace

extern "C" int dd_solve_noalloc(const dd_batch* batch, const dd_voltages* volts,
                                const dd_opts* opts, double* J, uint8_t* converged,
                                int32_t* iterations, int32_t* lane_status, int32_t* lane_steps,
                                void* stream) {
  size_t need = 0;
  if (dd_workspace_bytes(batch, &need) != DD_OK) return DD_ERR_ARGS;
  if (need > (size_t)DD_NOALLOC_SCRATCH_BYTES) return DD_ERR_SCRATCH;
  const int dst = dd::device_status();
  if (dst != DD_OK) return dst;
  void* scratch = noalloc_scratch_ptr();
  if (!scratch) return DD_ERR_DEVICE;
  return dd_solve(batch, volts, opts, J, converged, iterations, lane_status, lane_steps, scratch,
                  (size_t)DD_NOALLOC_SCRATCH_BYTES, stream);
}
