// What jaxdd's `solve_states` reports of each solution (`_observed`, src/jaxdd/batch.py:1009-1030;
// `solve_states`, 1165-1191), from the checkpoints `dd_solve_states` wrote: the profiles on all
// NP + 2 points (V, n, p, the quasi-Fermi level splitting V_T ln(n p / n_i^2), anions, cations)
// and the radiative measures of direct recombination: implied V_oc = V_T ln(rad / rad_0) and
// PLQY = (rad - rad_0) / gen, with rad = sum vol k n p, rad_0 = sum vol k n_i^2,
// gen = G_frac sum vol G over the interior points' control volumes vol = fac / (L h_m h_p)
// (`solver._volumes`, solver.py:1952-1954). The contacts' states are the contacts' values at the
// voltage; the ions' boundary points are their neighbours' (`_ions_on_grid`, solver.py:2096-2102).
// A device whose ions are frozen after its pre-bias reports the frozen densities, recomputed
// here from the pre-bias checkpoint as the solve froze them.
//
// One thread per (device, voltage): every profile is written lane-interleaved,
// [voltage][node][lane], so a warp's writes of one node are contiguous.
#include <cuda_runtime.h>
#include <stdint.h>

#include "dd_launch.h"
#include "dd_layout.h"
#include "dd_physics.cuh"
#include "../../include/jaxdd_b200.h"

namespace dd {
namespace obs {

struct Args {
  int B, Bp, npmax, ka;
  const double* S;
  const double* C;
  const double* IFt;
  const double* V;
  const int* voff;
  const int* vcnt;
  const double* states;
  const double* state_logs;
  const double* prebias;
  const double* prebias_logs;
  int nv_max;
  double *oV, *on, *op, *oq, *oa, *oc, *ovoc, *oplqy;
};

template <int K>
__global__ void __launch_bounds__(64) observe_kernel(Args a) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int l = (int)(t % a.Bp);
  const int j = (int)(t / a.Bp);
  if (l >= a.B || j >= a.nv_max || j >= a.vcnt[l]) return;
  Lane L;
  L.S = a.S; L.C = a.C; L.IFt = a.IFt; L.Bp = a.Bp; L.l = l; L.ka = a.ka; L.K = K;
  L.Vt = L.sc(C_VT); L.iVt = 1.0 / L.Vt; L.L = L.sc(C_L);
      L.gfrac = L.sc(C_GFRAC);
  L.NP = (int)L.sc(C_NP);
  L.share = 1.0; L.frozen = false; L.FX = nullptr; L.CD = nullptr; L.ybuf = 0;
  const int NP = L.NP;
  const size_t nodes = (size_t)a.npmax + 2;
  const double Vint = a.V[a.voff[l] + j];
  const bool frozen = L.sc(C_PRECOND) > 0.0 && L.sc(C_FIXIONS) > 0.0;
  double logs[K], plogs[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    logs[k] = a.state_logs[((size_t)j * DD_MAXK + k) * a.Bp + l];
    plogs[k] = a.prebias_logs[(size_t)k * a.Bp + l];
  }
  const double* ys = a.states + (size_t)j * nodes * 3 * a.Bp;
  auto out = [&](double* o, int k) -> double& { return o[((size_t)j * nodes + k) * a.Bp + l]; };
  double rad = 0.0, rad0 = 0.0, gen = 0.0, a1 = 0.0, c1 = 0.0, aN = 0.0, cN = 0.0;
  for (int k = 0; k <= NP + 1; ++k) {
    Pt P;
    if (k == 0) contact(L, 0, Vint, P);
    else if (k == NP + 1) contact(L, 1, Vint, P);
    else {
      P.V = ys[((size_t)k * 3 + 0) * a.Bp + l];
      P.lnn = ys[((size_t)k * 3 + 1) * a.Bp + l];
      P.lnp = ys[((size_t)k * 3 + 2) * a.Bp + l];
    }
    const double n = exp(P.lnn), p = exp(P.lnp), ni2 = L.st(k, S_NI2);
    out(a.oV, k) = P.V;
    out(a.on, k) = n;
    out(a.op, k) = p;
    out(a.oq, k) = L.Vt * log(n * p / ni2);
    if (k >= 1 && k <= NP) {
      // ions: mobile ones Boltzmann in V, frozen ones as the pre-bias left them
      double an, ca;
      if (frozen) {
        Pt Q0;
        Q0.V = a.prebias[((size_t)k * 3) * a.Bp + l];
        Q0.sl = slots_at(L, k);
        an = L.st(k, S_AFIX) + (Q0.sl.a >= 0 ? exp(plogs[Q0.sl.a] + Q0.V * L.iVt) : 0.0);
        ca = L.st(k, S_CFIX) + (Q0.sl.c >= 0 ? exp(plogs[L.ka + Q0.sl.c] - Q0.V * L.iVt) : 0.0);
      } else {
        const Slots sl = slots_at(L, k);
        an = L.st(k, S_AFIX) + (sl.a >= 0 ? exp(logs[sl.a] + P.V * L.iVt) : 0.0);
        ca = L.st(k, S_CFIX) + (sl.c >= 0 ? exp(logs[L.ka + sl.c] - P.V * L.iVt) : 0.0);
      }
      out(a.oa, k) = an;
      out(a.oc, k) = ca;
      if (k == 1) { a1 = an; c1 = ca; }
      if (k == NP) { aN = an; cN = ca; }
      const double vol = L.st(k, S_FAC) / (L.L * L.st(k - 1, S_H) * L.st(k, S_H));
      const double kd = L.st(k, S_KD);
      rad += vol * kd * n * p;
      rad0 += vol * kd * ni2;
      gen += vol * L.st(k, S_G);
    }
  }
  out(a.oa, 0) = a1; out(a.oc, 0) = c1;
  out(a.oa, NP + 1) = aN; out(a.oc, NP + 1) = cN;
  gen *= L.gfrac;
  a.ovoc[(size_t)j * a.Bp + l] = rad0 > 0.0 ? L.Vt * log(rad / rad0) : NAN;
  a.oplqy[(size_t)j * a.Bp + l] = gen > 0.0 ? (rad - rad0) / gen : NAN;
}

}  // namespace obs
}  // namespace dd

extern "C" int dd_observables(const dd_batch* batch, const dd_voltages* volts,
                              const double* states, const double* state_logs,
                              const double* prebias, const double* prebias_logs, int nv_max,
                              double* V, double* n, double* p, double* qfls, double* anion,
                              double* cation, double* implied_voc, double* plqy, void* stream) {
  if (!batch || !batch->stat || !batch->scal || !batch->iface || !volts || !volts->v ||
      !volts->offset || !volts->count || !states || !state_logs || !prebias || !prebias_logs ||
      nv_max < 1 || !V || !n || !p || !qfls || !anion || !cation || !implied_voc || !plqy)
    return DD_ERR_ARGS;
  if (batch->n_lanes < 1 || batch->lane_stride < batch->n_lanes || batch->lane_stride % 32 != 0 ||
      batch->np_max < 3 || batch->k_anion < 1 || batch->k_cation < 1 ||
      batch->k_anion + batch->k_cation > dd::DD_MAXK)
    return DD_ERR_ARGS;
  dd::obs::Args a{};
  a.B = batch->n_lanes; a.Bp = batch->lane_stride; a.npmax = batch->np_max; a.ka = batch->k_anion;
  a.S = batch->stat; a.C = batch->scal; a.IFt = batch->iface;
  a.V = volts->v; a.voff = volts->offset; a.vcnt = volts->count;
  a.states = states; a.state_logs = state_logs; a.prebias = prebias; a.prebias_logs = prebias_logs;
  a.nv_max = nv_max;
  a.oV = V; a.on = n; a.op = p; a.oq = qfls; a.oa = anion; a.oc = cation; a.ovoc = implied_voc;
  a.oplqy = plqy;
  const long T = (long)batch->lane_stride * nv_max;
  const dim3 block(64), grid((unsigned)((T + 63) / 64));
  const int st = dd::device_status();
  if (st != DD_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  return batch->k_anion + batch->k_cation <= 2
             ? dd::launch(dd::obs::observe_kernel<2>, grid, block, 0, s, a)
             : dd::launch(dd::obs::observe_kernel<4>, grid, block, 0, s, a);
}
