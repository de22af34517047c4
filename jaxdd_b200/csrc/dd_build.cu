// Device building on the GPU: the packed record (dd_layout.h) of many devices of one stack
// structure from per-device layer parameters, as jaxdd's `device_tree(structure, params)`
// builds them in JAX for parameter sweeps (src/jaxdd/batch.py:142-148 over
// `device.device_arrays`, device.py:877-1063): the grid's points per layer held fixed, the
// spacings scaled by the thicknesses, every array of the steady solve from the layers' values.
//
// The formulas are those of this package's host builder and packer (jaxdd_b200/device.py
// `build_device`, jaxdd_b200/batch.py `_pack_one`), restated per node in the same order of
// operations, so that a record built here equals the host's but for the two sums NumPy takes
// pairwise (the spacings' sum and the current scale's integral; a few units in the last place).
//
// One thread per device: it walks the device's nodes once for the grid, once for the fields;
// every write of one (node, field) by a warp is 32 consecutive lanes.
#include <cuda_runtime.h>
#include <stdint.h>

#include "dd_launch.h"
#include "dd_layout.h"
#include "../../include/jaxdd_b200.h"

namespace dd {
namespace bld {

constexpr double Q = 1.6022e-19, K_B = 1.3807e-23, EPS_0 = 8.8542e-12;

struct Args {
  dd_structure st;
  const double* P;   // [layers][DD_LF][n]
  const double* D;   // [DD_DF][n]
  int n, Bp, npmax, ka, kc;
  double* S;
  double* C;
  double* I;
  double* y0;
  double* h;         // scratch [np+2][n]: the spacings
};

__device__ __forceinline__ double par(const Args& a, int layer, int f, int l) {
  return a.P[((size_t)layer * DD_LF + f) * a.n + l];
}

__global__ void __launch_bounds__(64) build_kernel(Args a) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= a.n) return;
  const dd_structure& st = a.st;
  const int NP = st.np, nl = st.n_layers;
  const int Bp = a.Bp;
  auto S = [&](int k, int f) -> double& { return a.S[((size_t)k * DD_NF + f) * Bp + l]; };
  auto C = [&](int f) -> double& { return a.C[(size_t)f * Bp + l]; };
  auto H = [&](int k) -> double& { return a.h[(size_t)k * a.n + l]; };
  auto lid = [&](int k) { return (int)st.lid[k]; };
  const double T = a.D[(size_t)DD_D_T * a.n + l];
  const double Vt = K_B * T / Q;
  // the total thickness, summed as Python adds floats (Neumaier)
  double s = 0.0, c = 0.0;
  for (int j = 0; j < nl; ++j) {
    const double v = par(a, j, DD_L_L, l);
    const double t = s + v;
    c += fabs(s) >= fabs(v) ? (s - t) + v : (v - t) + s;
    s = t;
  }
  const double total = s + c;
  // spacings: each layer's raw spacings scaled to its thickness, then the three around each join
  // set to their mean
  for (int k = 0; k <= NP + 1; ++k) {
    const int j = lid(k);
    H(k) = st.raw[k] * (par(a, j, DD_L_L, l) / (total * st.norm[j]));
  }
  for (int j = 1; j < nl; ++j) {
    const int m = st.i0[j];
    const double mean = (H(m) + H(m - 1) + H(m - 2)) / 3.0;
    H(m - 2) = mean; H(m - 1) = mean; H(m) = mean;
  }
  // per node
  const double Nc0 = par(a, lid(0), DD_L_NC, l), Ec0 = par(a, lid(0), DD_L_EC, l);
  const double Ev0 = par(a, lid(0), DD_L_EV, l);
  double ncmax = 0.0;
  double x = 0.0, xprev = 0.0;
  double genh = 0.0, hsum_g = 0.0;
  for (int k = 0; k <= NP + 1; ++k) {
    const int j = lid(k);
    const double h = H(k);
    const bool inner = k >= 1 && k <= NP;
    const double Ec = par(a, j, DD_L_EC, l), Ev = par(a, j, DD_L_EV, l), Nc = par(a, j, DD_L_NC, l);
    ncmax = fmax(ncmax, Nc);
    const double dos = Vt * log(Nc / Nc0);
    S(k, S_OFFN) = Ec - Ec0 + dos;
    S(k, S_OFFP) = Ev - Ev0 - dos;
    const bool at_iface = st.at_iface[k] != 0;
    const double mun = at_iface ? (total * h) * par(a, j, DD_L_NUN, l) / Vt : par(a, j, DD_L_MUN, l);
    const double mup = at_iface ? (total * h) * par(a, j, DD_L_NUP, l) / Vt : par(a, j, DD_L_MUP, l);
    S(k, S_MUN) = mun;
    S(k, S_MUP) = mup;
    S(k, S_H) = h;
    // x and its differences as the host's cumulative sum makes them: the product and the sum
    // rounded apart (a fused multiply-add would differ in the last place, and the differences
    // of neighbouring x magnify that where the spacing is fine)
    if (k >= 1) x = __dadd_rn(xprev, __dmul_rn(total, H(k - 1)));
    if (k >= 1 && k <= NP) S(k - 1, S_DX) = x - xprev;
    xprev = x;
    const double ni = Nc * exp(-0.5 * (Ev - Ec) / Vt);
    S(k, S_KD) = inner ? par(a, j, DD_L_KD, l) : 0.0;
    S(k, S_NI2) = ni * ni;
    const double Nt = par(a, j, DD_L_NTB, l);
    const bool trap = inner && Nt != 0.0;
    const double Et = par(a, j, DD_L_ETB, l);
    S(k, S_NT) = trap ? Nt : 0.0;
    S(k, S_CNT) = trap ? par(a, j, DD_L_CNB, l) : 0.0;
    S(k, S_CPT) = trap ? par(a, j, DD_L_CPB, l) : 0.0;
    S(k, S_NT0) = trap ? Nc * exp((Ec - Et) / Vt) : 0.0;
    S(k, S_PT0) = trap ? Nc * exp((Et - Ev) / Vt) : 0.0;
    const double G = inner ? par(a, j, DD_L_G, l) : 0.0;
    S(k, S_G) = G;
    if (k <= NP) { genh += h * G; hsum_g += h; }
    S(k, S_ASLOT) = st.aslot[j];
    S(k, S_CSLOT) = st.cslot[j];
    S(k, S_IFK) = st.ifk[k];
    if (inner) {
      const double hm = H(k - 1), hp = h, w = hp + hm, L2 = total * total;
      const double ei = par(a, j, DD_L_EPS, l) * EPS_0;
      const double em = par(a, lid(k - 1), DD_L_EPS, l) * EPS_0;
      S(k, S_FACU) = 2 * ei / (hp * w * L2);
      S(k, S_FACL) = 2 * ei / (hm * w * L2) - (ei - em) / (hm * hm * L2);
      S(k, S_FACM) = (ei - em) / (hm * hm * L2) - 2 * ei * (1 / (hp * w * L2) + 1 / (hm * w * L2));
      S(k, S_FAC) = 0.5 * L2 * hp * hm * w;
      S(k, S_SP) = 1.0 / (Q * Nc);
      S(k, S_SC) = 1.0 / (fmax(mun, mup) * Vt * Nc * hp);
      S(k, S_DOP) = par(a, j, DD_L_NA, l) - par(a, j, DD_L_ND, l);
      S(k, S_AFIX) = st.afixed[j] ? par(a, j, DD_L_NAN, l) : 0.0;
      S(k, S_CFIX) = st.cfixed[j] ? par(a, j, DD_L_NCA, l) : 0.0;
    } else {
      S(k, S_FACU) = 0.0; S(k, S_FACL) = 0.0; S(k, S_FACM) = 0.0; S(k, S_FAC) = 0.0;
      S(k, S_SP) = 1.0; S(k, S_SC) = 1.0; S(k, S_DOP) = 0.0;
      S(k, S_AFIX) = 0.0; S(k, S_CFIX) = 0.0;
    }
  }
  S(NP, S_DX) = 0.0;
  S(NP + 1, S_DX) = 0.0;
  // the contacts: flat-band where their layer's doping sets them
  const int jl = 0, jr = nl - 1;
  auto sfb = [&](int j) {
    const double net = par(a, j, DD_L_NA, l) - par(a, j, DD_L_ND, l);
    const double Nc = par(a, j, DD_L_NC, l);
    if (net > 0) return par(a, j, DD_L_EV, l) - Vt * log(Nc / fabs(net));
    if (net < 0) return par(a, j, DD_L_EC, l) + Vt * log(Nc / fabs(net));
    return 0.5 * (par(a, j, DD_L_EC, l) + par(a, j, DD_L_EV, l));
  };
  const double WL = st.sfb_left ? sfb(jl) : a.D[(size_t)DD_D_WL * a.n + l];
  const double WR = st.sfb_right ? sfb(jr) : a.D[(size_t)DD_D_WR * a.n + l];
  const double NcR = par(a, jr, DD_L_NC, l), EcR = par(a, jr, DD_L_EC, l), EvR = par(a, jr, DD_L_EV, l);
  const double V0 = 0.5 * (-WL + WR), VL = 0.5 * (WL - WR);
  C(C_VT) = Vt;
  C(C_L) = total;
  C(C_V0) = V0;
  C(C_VL) = VL;
  C(C_LEFT) = st.left_elec;
  C(C_LNNL) = log(Nc0 * exp(-(WL - Ec0) / Vt));
  C(C_LNPL) = log(Nc0 * exp((WL - Ev0) / Vt));
  C(C_LNNR) = log(NcR * exp(-(WR - EcR) / Vt));
  C(C_LNPR) = log(NcR * exp(-(EvR - WR) / Vt));
  const double generated = Q * total * genh / hsum_g;
  C(C_JSCALE) = fmax(generated, 1.0);
  const double Rsh = a.D[(size_t)DD_D_RSHUNT * a.n + l];
  C(C_GSHUNT) = Rsh > 0 ? 1.0 / Rsh : 0.0;
  C(C_PRECOND) = st.pre_cond;
  C(C_VPRE) = a.D[(size_t)DD_D_VPRE * a.n + l];
  C(C_FIXIONS) = st.fix_ions;
  C(C_GFRAC) = a.D[(size_t)DD_D_GFRAC * a.n + l];
  C(C_NFLOOR) = 1e-12 * ncmax;
  C(C_NP) = NP;
  C(C_CURRDIFF) = st.curr_diff;
  C(C_HSUM) = hsum_g;
  C(C_MID) = st.mid;
  for (int k = 0; k < a.ka + a.kc; ++k) C(C_TOT0 + k) = 0.0;
  for (int j = 0; j < nl; ++j) {
    const double Lj = par(a, j, DD_L_L, l);
    if (st.aslot[j] >= 0) C(C_TOT0 + (int)st.aslot[j]) += Lj * par(a, j, DD_L_NAN, l);
    if (st.cslot[j] >= 0) C(C_TOT0 + a.ka + (int)st.cslot[j]) += Lj * par(a, j, DD_L_NCA, l);
  }
  // interface traps: the rows of the trapped joins
  for (int r = 0; r < DD_MAXIF; ++r)
    for (int f = 0; f < DD_NIF; ++f) a.I[((size_t)r * DD_NIF + f) * Bp + l] = 0.0;
  for (int j = 0; j < nl - 1; ++j) {
    const int r = st.iface_row[j];
    if (r < 0) continue;
    const int e = st.i1[j];
    const double Et = par(a, j, DD_L_ETI, l);
    auto put = [&](int f, double v) { a.I[((size_t)r * DD_NIF + f) * Bp + l] = v; };
    const double kind = st.iface_kind[j];
    put(I_NT, par(a, j, DD_L_NTI, l));
    put(I_CN, par(a, j, DD_L_CNI, l));
    put(I_CP, par(a, j, DD_L_CPI, l));
    put(I_NT0LO, par(a, j, DD_L_NC, l) * exp((par(a, j, DD_L_EC, l) - Et) / Vt));
    put(I_PT0LO, par(a, j, DD_L_NC, l) * exp((Et - par(a, j, DD_L_EV, l)) / Vt));
    put(I_NT0HI, par(a, j + 1, DD_L_NC, l) * exp((par(a, j + 1, DD_L_EC, l) - Et) / Vt));
    put(I_PT0HI, par(a, j + 1, DD_L_NC, l) * exp((Et - par(a, j + 1, DD_L_EV, l)) / Vt));
    put(I_IW, 1.0 / (0.5 * total * (0.5 * H(e + 1) + H(e) + 0.5 * H(e - 1))));
    put(I_CHARGE, fabs(kind));
    put(I_CWE, kind == 1.0 ? 1.0 : 0.0);
  }
  // the start: SIMsalabim's linear potential and Fermi level at the first voltage
  if (a.y0) {
    const double first = a.D[(size_t)DD_D_FIRST * a.n + l];
    const double e = st.left_elec;
    double xx = 0.0;
    for (int k = 0; k <= NP + 1; ++k) {
      if (k >= 1) xx = __dadd_rn(xx, __dmul_rn(total, H(k - 1)));
      const int j = lid(k);
      const double Ec = par(a, j, DD_L_EC, l), Ev = par(a, j, DD_L_EV, l), Nc = par(a, j, DD_L_NC, l);
      const double ni = Nc * exp(-0.5 * (Ev - Ec) / Vt);
      const double V = V0 + 0.5 * e * first + xx * (VL - V0 - e * first) / total;
      const double EF = WL - xx * (WL - WR) / total;
      const double lnn = log(Nc) - (EF - Ec) / Vt;
      a.y0[((size_t)k * 3 + 0) * Bp + l] = V;
      a.y0[((size_t)k * 3 + 1) * Bp + l] = lnn;
      a.y0[((size_t)k * 3 + 2) * Bp + l] = 2 * log(ni) - lnn;
    }
  }
}

}  // namespace bld
}  // namespace dd

extern "C" int dd_build(const dd_structure* structure, const double* layer_params,
                        const double* device_params, int n_devices, int lane_stride,
                        int k_anion, int k_cation, double* stat, double* scal, double* iface,
                        double* y0, void* workspace, size_t workspace_bytes, void* stream) {
  if (!structure || !layer_params || !device_params || n_devices < 1 ||
      lane_stride < n_devices || lane_stride % 32 != 0 || !stat || !scal || !iface || !workspace)
    return DD_ERR_ARGS;
  const dd_structure& st = *structure;
  if (st.np < 3 || st.n_layers < 1 || st.n_layers > DD_MAXLAYERS || !st.lid || !st.raw ||
      !st.norm || !st.i0 || !st.i1 || !st.at_iface || !st.ifk || !st.aslot || !st.cslot ||
      !st.afixed || !st.cfixed || !st.iface_row || !st.iface_kind || k_anion < 1 ||
      k_cation < 1 || k_anion + k_cation > dd::DD_MAXK)
    return DD_ERR_ARGS;
  if (workspace_bytes < (size_t)(st.np + 2) * n_devices * sizeof(double)) return DD_ERR_WORKSPACE;
  dd::bld::Args a{};
  a.st = st;
  a.P = layer_params; a.D = device_params; a.n = n_devices; a.Bp = lane_stride;
  a.npmax = st.np; a.ka = k_anion; a.kc = k_cation;
  a.S = stat; a.C = scal; a.I = iface; a.y0 = y0;
  a.h = static_cast<double*>(workspace);
  const int dst = dd::device_status();
  if (dst != DD_OK) return dst;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  return dd::launch(dd::bld::build_kernel, dim3((n_devices + 63) / 64), dim3(64), 0, s, a);
}
