// Packed batch layout shared by the host packer (jaxdd_b200/batch.py) and the kernels.
//
// Every array is lane-interleaved: the lane (one device) is the fastest index, so a warp's
// access to one (node, field) is 32 consecutive words. Field indices below are the second
// fastest; nodes (0 … NP+1 of the device's grid, contacts included) the slowest.
#pragma once

namespace dd {

// Per-node static fields, stat[(node * DD_NF + field) * lane_stride + lane].
// "point k" fields belong to grid point k; "edge k" fields to the interval (k, k+1);
// "row k" fields to the equations of interior point k (zero on the contacts).
enum StaticField {
  S_OFFN = 0,   // point: Vgn - V (band offset and DOS term), V
  S_OFFP,       // point: Vgp - V, V
  S_MUN,        // edge: electron mobility of the interval (interface: its transfer mobility)
  S_MUP,        // edge: hole mobility
  S_H,          // edge: (x[k+1] - x[k]) / L as the grid defines it
  S_DX,         // edge: x[k+1] - x[k] (0 for k = NP)
  S_FACL,       // row: Poisson stencil, left
  S_FACM,       // row: Poisson stencil, centre
  S_FACU,       // row: Poisson stencil, right
  S_FAC,        // row: continuity control-volume factor 0.5 L^2 h[k] h[k-1] (h[k] + h[k-1])
  S_SP,         // row: Poisson row scale 1 / (q N_c)
  S_SC,         // row: continuity row scale 1 / (max(mu_n, mu_p) V_T N_c h[k])
  S_DOP,        // row: N_A - N_D
  S_KD,         // point: direct recombination coefficient (0 on the contacts)
  S_NI2,        // point: n_i^2
  S_NT,         // point: bulk trap density (SRH, one neutral level)
  S_CNT,        // point: electron capture coefficient
  S_CPT,        // point: hole capture coefficient
  S_NT0,        // point: SRH n_1
  S_PT0,        // point: SRH p_1
  S_G,          // point: generation at G_frac = 1
  S_ASLOT,      // point: anion slot index of the point's mobile region, -1 none
  S_CSLOT,      // point: cation slot index (counted from 0 within the cations), -1 none
  S_AFIX,       // row: fixed anion density
  S_CFIX,       // row: fixed cation density
  S_IFK,        // edge: -2 no layer interface, -1 interface without traps, >= 0 trap table row
  DD_NF
};

// Per-lane scalars, scal[field * lane_stride + lane].
enum ScalarField {
  C_VT = 0, C_L, C_V0, C_VL, C_LEFT, C_LNNL, C_LNPL, C_LNNR, C_LNPR,
  C_JSCALE, C_GSHUNT, C_PRECOND, C_VPRE, C_FIXIONS, C_GFRAC, C_NFLOOR, C_NP, C_CURRDIFF,
  C_HSUM,       // sum of h over the NP + 1 intervals
  C_MID,        // the row where the two halves of the twisted sweep meet (no interface within
                // one interval of it)
  C_TOT0,       // slot totals follow: C_TOT0 + k, k < K (anion slots first)
  DD_NS_BASE = C_TOT0
};

// Interface-trap table, iface[(row * DD_NIF + field) * lane_stride + lane].
enum IfaceField {
  I_NT = 0, I_CN, I_CP, I_NT0LO, I_PT0LO, I_NT0HI, I_PT0HI, I_IW, I_CHARGE, I_CWE, DD_NIF
};

constexpr int DD_MAXIF = 4;   // interface-trap rows per lane
constexpr int DD_MAXK = 4;    // ion slots (anion + cation regions)
constexpr int DD_NBUF = 4;    // state buffers per lane: iterate, carry, previous carry, start

}  // namespace dd
