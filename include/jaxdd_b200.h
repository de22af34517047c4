/* jaxdd_b200 — C ABI of the batched steady-state drift-diffusion solve on sm_100a.
 *
 * The drop-in boundary for jaxdd's batched J-V path. jaxdd itself has no native layer: its
 * solve is one jitted JAX program (`_solve_batch`, jaxdd src/jaxdd/batch.py:1033-1047) whose
 * only hand-written kernel is the Pallas block sweep (`block_sweep`, src/jaxdd/sweep.py:313-330).
 * These entry points are what an XLA FFI custom call (or ctypes / a torch extension) binds in
 * its place: plain pointers and sizes, caller-owned device buffers, stream-ordered, no host
 * synchronisation, no allocation (scratch comes from `dd_workspace_bytes`).
 *
 * Layout: every array is lane-interleaved (one lane = one device; lane fastest), see
 * jaxdd_b200/csrc/dd_layout.h for the field indices. The host packer that writes it is
 * jaxdd_b200/batch.py (`prepare`).
 *
 * Errors: a nonzero status for invalid arguments or a failed launch. Non-convergence is never
 * an error: it is reported per (device, voltage) in `converged`, as jaxdd reports it
 * (docs/solver.md "Convergence"; batch.py:1006).
 */
#ifndef JAXDD_B200_H
#define JAXDD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define DD_OK 0
#define DD_ERR_ARGS 1       /* a size, pointer or option out of range */
#define DD_ERR_WORKSPACE 2  /* workspace smaller than dd_workspace_bytes */
#define DD_ERR_LAUNCH 3     /* the CUDA launch failed (the launch's own error) */
#define DD_ERR_DEVICE 4     /* no sm_100 device current */
#define DD_ERR_SCRATCH 5    /* dd_solve_noalloc: the batch needs more scratch than
                               DD_NOALLOC_SCRATCH_BYTES */

/* Size of dd_solve_noalloc's fixed scratch array (64 MiB per device). */
#define DD_NOALLOC_SCRATCH_BYTES (64u << 20)

/* Per-lane status written by dd_solve (lane_status). */
#define DD_LANE_OK 0
#define DD_LANE_PREBIAS_FAILED 1 /* solve_jv mode: the pre-bias did not converge
                                    (jaxdd solver.py:2228-2229 raises RuntimeError) */

/* A packed batch (device pointers). Mirrors the pytree `prepare` returns
 * (jaxdd batch.py:151-223), in the layout of dd_layout.h. */
typedef struct dd_batch {
  int32_t n_lanes;     /* devices in the batch */
  int32_t lane_stride; /* >= n_lanes, a multiple of 32 */
  int32_t np_max;      /* the largest grid size NP of any lane (interior points) */
  int32_t k_anion;     /* anion slots (mobile regions), >= 1 */
  int32_t k_cation;    /* cation slots, >= 1; k_anion + k_cation <= 4 */
  const double* stat;  /* [(np_max + 2)][DD_NF][lane_stride] */
  const double* scal;  /* [DD_NS_BASE + k_anion + k_cation][lane_stride] */
  const double* iface; /* [DD_MAXIF][DD_NIF][lane_stride] */
  const double* y0;    /* [(np_max + 2)][3][lane_stride]: (V, ln n, ln p) start at the first voltage */
} dd_batch;

/* Each lane's voltages (internal, V), flat: lane l's are v[offset[l] ... offset[l]+count[l]).
 * Ascending in DD_MODE_BATCH (solve_batch sorts them, batch.py:1043-1045); in the caller's
 * order in DD_MODE_JV. Outputs J/converged/iterations use the same flat positions. */
typedef struct dd_voltages {
  const double* v;
  const int32_t* offset;
  const int32_t* count;
} dd_voltages;

#define DD_MODE_BATCH 0 /* jaxdd batch.solve_batch: outward scan, extrapolated starts */
#define DD_MODE_JV 1    /* jaxdd solver.solve_jv: caller's order, each from the last solution */

#define DD_BERNOULLI_EXACT 0 /* solver.bernoulli (solver.py:95-105) */
#define DD_BERNOULLI_SIMSS 1 /* solver.bernoulli_simss (solver.py:108-121) */

#define DD_PRECISION_FP64 0  /* everything in FP64: the only precision dd_solve accepts */
#define DD_PRECISION_MIXED 1 /* FP32 Jacobian and block sweep, FP64 residual, update and current:
                                refused (DD_ERR_ARGS). Measured: an FP32 sweep (each node's rows
                                and unknowns scaled first) contracts Newton's step only linearly;
                                even used per device only while the last step exceeds 0.1, it
                                takes 9 % more steps and changes 3 of 3,904 converged flags of the
                                drawn J-V curves (oracle.mixed_sweep), so it can neither give
                                jaxdd's flags nor be 2x faster. */

typedef struct dd_opts {
  double tol;         /* Newton's step tolerance (solve_batch tol, default 1e-10) */
  int32_t max_iter;   /* Newton steps per voltage (60 batch, 200 jv) */
  int32_t start_iter; /* Poisson / start / pre-bias cap (= max_iter in jaxdd) */
  int32_t strict;     /* 1: only tol or the round-off floor stop Newton (batch.py:815-816) */
  int32_t bernoulli;  /* DD_BERNOULLI_* */
  int32_t mode;       /* DD_MODE_* */
  int32_t precision;  /* DD_PRECISION_* */
  int32_t reserved;
} dd_opts;

/* Scratch bytes dd_solve needs for this batch (four state buffers, the frozen-ion profile,
 * the sweep's c'/d' per node, the work queue's counter). */
int dd_workspace_bytes(const dd_batch* batch, size_t* bytes);

/* The J-V curves of a batch: jaxdd's solve_batch (DD_MODE_BATCH; batch.py:1136-1162, one pass
 * at max_iter, which gives what its two passes give) or solve_jv (DD_MODE_JV; solver.py:2041-2060)
 * for every lane. J (A/m^2, SIMsalabim's sign, the shunt's current added), converged (0/1) and
 * iterations at each flat voltage position; lane_status per lane; lane_steps (may be NULL)
 * [3][lane_stride] the steps each lane took in all: Newton steps with the ions' border (mobile
 * ions), Newton steps without it, Poisson steps. Asynchronous on `stream` (a cudaStream_t,
 * NULL the legacy default stream). A batch of more devices than the GPU holds at once is solved
 * from a work queue (each pair of threads takes the next device when its own is done, in lane
 * order) unless dd_tune chose otherwise for its shape; the results do not depend on it. */
int dd_solve(const dd_batch* batch, const dd_voltages* volts, const dd_opts* opts, double* J,
             uint8_t* converged, int32_t* iterations, int32_t* lane_status, int32_t* lane_steps,
             void* workspace, size_t workspace_bytes, void* stream);

/* Launch forms of the solve (threads per block; the work queue for a batch larger than the GPU
 * holds at once, or one pair of threads per device) that dd_tune chooses among. */
#define DD_SOLVE_FORMS 4

/* The solve's autotuner: runs dd_solve on this batch once in each launch form (synchronising
 * `stream` to time each with events), keeps the fastest for later dd_solve and dd_solve_states
 * calls in this process on batches of the same shape (device, ion slots, np_max, lane count
 * within a factor of two), and returns its index in `form` and, unless NULL, each form's time
 * in `times_ms` [DD_SOLVE_FORMS]. The outputs are dd_solve's (every form gives the same). Untuned
 * shapes take form 0. No counterpart in the reference, which compiles one XLA program per
 * shape. */
int dd_tune(const dd_batch* batch, const dd_voltages* volts, const dd_opts* opts, double* J,
            uint8_t* converged, int32_t* iterations, int32_t* lane_status, int32_t* lane_steps,
            void* workspace, size_t workspace_bytes, void* stream, int32_t* form,
            float* times_ms);

/* dd_solve that also keeps what differentiating the curves needs (jaxdd keeps the same under
 * `jax.checkpoint`: the converged solution per voltage, `_tangent`, batch.py:676-680): for each
 * lane's voltage j (its j-th in `volts`, j < nv_max) the final iterate `states`
 * [nv_max][np_max+2][3][lane_stride] (interior nodes written) and its ion normalisations
 * `state_logs` [nv_max][DD_MAXK][lane_stride]; and the solution at the pre-bias (or first)
 * voltage, before any freeze, `prebias` [np_max+2][3][lane_stride], `prebias_logs`
 * [DD_MAXK][lane_stride]. Results otherwise those of dd_solve, in either mode: DD_MODE_JV with
 * one voltage is jaxdd's `solve_state` (solver.py:2063-2093) once dd_observables has read the
 * checkpoint; dd_adjoint (which reads no mode) is used and tested on DD_MODE_BATCH's. */
int dd_solve_states(const dd_batch* batch, const dd_voltages* volts, const dd_opts* opts,
                    double* J, uint8_t* converged, int32_t* iterations, int32_t* lane_status,
                    int32_t* lane_steps, double* states, double* state_logs, double* prebias,
                    double* prebias_logs, int nv_max, void* workspace, size_t workspace_bytes,
                    void* stream);

/* Scratch bytes dd_adjoint needs for this batch. */
int dd_adjoint_workspace_bytes(const dd_batch* batch, size_t* bytes);

/* The adjoint of dd_solve_states: given J_bar (dL/dJ at every flat voltage position), the
 * gradient of L with respect to the packed inputs — stat_bar [np_max+2][DD_NF][lane_stride],
 * scal_bar [DD_NS_BASE+DD_MAXK][lane_stride], iface_bar [DD_MAXIF][DD_NIF][lane_stride], each
 * laid out as its input — by implicit differentiation at the checkpointed solutions: jaxdd's
 * `_converged_jvp` / `_tangent` in reverse mode (batch.py:661-737), one transposed bordered solve
 * per converged voltage, plus one at the pre-bias for devices whose ions are frozen after it.
 * `converged`, `states`, `state_logs`, `prebias`, `prebias_logs`, `nv_max` as dd_solve_states
 * wrote them for the same batch and voltages; not-converged voltages contribute nothing.
 * Derivatives are given for every continuous input the residual, the ions' constraints and the
 * integral current read (stencils, mobilities, spacings, offsets, doping, recombination
 * parameters, generation, fixed ions; length, contacts, ion totals, shunt, generation factor,
 * pre-bias voltage; interface trap density and width); the thermal voltage, the row scales' own
 * inputs beyond SP/SC, the interface capture coefficients and trap levels, and the
 * integer fields (slots, interface index) get none (zero). A device with the differential
 * current (`currDiffInt = 1`) gets NaN in scal_bar[C_VT] and nothing else. The outputs are
 * zeroed and written on `stream`. */
int dd_adjoint(const dd_batch* batch, const dd_voltages* volts, const dd_opts* opts,
               const uint8_t* converged, const double* J_bar, const double* states,
               const double* state_logs, const double* prebias, const double* prebias_logs,
               int nv_max, double* stat_bar, double* scal_bar, double* iface_bar,
               void* workspace, size_t workspace_bytes, void* stream);

/* What jaxdd's `solve_states` reports (batch.py:1009-1030, 1165-1191) of the checkpoints
 * dd_solve_states wrote: per lane and voltage j < min(count, nv_max) the profiles on all
 * np_max + 2 points — V, n, p, qfls = V_T ln(n p / n_i^2), anion, cation (frozen ions as the
 * pre-bias left them; the ions' boundary points their neighbours') — each laid out
 * [nv_max][np_max+2][lane_stride], and the implied V_oc and PLQY of direct recombination
 * [nv_max][lane_stride] (NaN where the device has none, or no generation). */
int dd_observables(const dd_batch* batch, const dd_voltages* volts, const double* states,
                   const double* state_logs, const double* prebias, const double* prebias_logs,
                   int nv_max, double* V, double* n, double* p, double* qfls, double* anion,
                   double* cation, double* implied_voc, double* plqy, void* stream);

/* Scratch bytes dd_admittance needs for this batch and n_freq frequencies. */
int dd_admittance_workspace_bytes(const dd_batch* batch, int n_freq, size_t* bytes);

/* The small-signal admittance Y = dJ/dV_int (S/m^2, SIMsalabim's sign) of every lane at each of
 * n_freq angular frequencies `laps` ([n_freq][2]: i omega as re, im), about the steady state
 * `state` ([np_max+2][3][lane_stride], e.g. dd_solve_states' checkpoint at the voltage `vint`
 * [lane_stride]): jaxdd's `_admittance` for devices without mobile ions (impedance.py:230-353):
 * one complex block-tridiagonal solve of (J + i omega M + the traps' occupations' own dynamics)
 * dy = -dF/dV per (lane, frequency) and the linearised current of a time step (control-volume
 * widths, each density's change, the displacement current; `eps` [np_max+2][lane_stride] the
 * permittivity at every point). Y [n_freq][2][lane_stride] (re, im). A batch with mobile ions
 * goes to dd_admittance_ions instead (the host routes it there): here k_anion and k_cation must
 * be 1 (DD_ERR_ARGS otherwise). `dt` 0: the continuous
 * response; dt > 0: what a transient sees through implicit Euler at steps of dt (jaxdd's
 * `solve_impedance(..., dt=)`, impedance.py:379-383): `laps` then (1 - e^(-i omega dt))/dt and
 * the traps' occupations those of their exact step (its mean in the rates, its end in the
 * charge). */
int dd_admittance(const dd_batch* batch, const double* state, const double* eps,
                  const double* vint, const double* laps, int n_freq, int bernoulli, double dt,
                  double* Y, void* workspace, size_t workspace_bytes, void* stream);

#define DD_NT 3 /* per-point record of the transient and the impedance with ions: permittivity,
                   anion and cation mobility */

/* Scratch bytes dd_admittance_ions needs for this batch and n_freq frequencies. */
int dd_admittance_ions_workspace_bytes(const dd_batch* batch, int n_freq, size_t* bytes);

/* dd_admittance for devices with free mobile ions (jaxdd `_admittance` with `ions`,
 * impedance.py:242-353): the ions are unknowns of their own, the 5x5 blocks of a time step of
 * dt = 1 s from the steady state (its traps at their steady occupation) with (i omega - 1) M
 * added on the diagonal, the traps' occupations' dynamics on the carriers' blocks, each ion
 * region's number kept by a border (`_ion_constraints_time`), and each region's ion current in
 * the linearised current. `state` [np_max+2][3][lane_stride] and `state_logs`
 * [DD_MAXK][lane_stride] the steady state (dd_solve_states' checkpoint at `vint`, the ions
 * Boltzmann's of those normalisations); `tstat` [np_max+2][DD_NT][lane_stride] the
 * permittivity and the ions' mobilities. Several regions of a species each keep their own
 * number (a slot each: k_anion + k_cation <= DD_MAXK, the border K columns wide); devices without
 * mobile ions are solved too (their ions' rows identities). The differential current
 * (`currDiffInt = 1`) is each interval's Scharfetter-Gummel flux's tangent, the ions' too.
 * Y [n_freq][2][lane_stride]; `dt` as dd_admittance's. */
int dd_admittance_ions(const dd_batch* batch, const double* state, const double* state_logs,
                       const double* tstat, const double* vint, const double* laps, int n_freq,
                       int bernoulli, double dt, double* Y, void* workspace,
                       size_t workspace_bytes, void* stream);

/* ---- Device building on the GPU (parameter sweeps) ------------------------------------------
 * The packed record of n devices of one stack structure from their parameters, as jaxdd's
 * `device_tree(structure, params)` (batch.py:142-148, device.py:877-1063) builds them for sweeps:
 * the points per layer fixed, the spacings scaled by the thicknesses. */
#define DD_MAXLAYERS 16

/* Per-layer parameters, layer_params[layer][DD_LF][n] (SI units, energies in eV). */
enum dd_layer_field {
  DD_L_L = 0, DD_L_EPS, DD_L_EC, DD_L_EV, DD_L_NC, DD_L_ND, DD_L_NA, DD_L_MUN, DD_L_MUP,
  DD_L_KD, DD_L_NTB, DD_L_ETB, DD_L_CNB, DD_L_CPB, DD_L_NUN, DD_L_NUP, DD_L_NTI, DD_L_ETI,
  DD_L_CNI, DD_L_CPI, DD_L_G, DD_L_NAN, DD_L_NCA, DD_LF
};
/* Per-device parameters, device_params[DD_DF][n]: temperature, work functions (unused where the
 * structure's contact is flat-band), generation factor, shunt resistance, pre-bias voltage, and
 * the first voltage the start state y0 is made for. */
enum dd_device_field {
  DD_D_T = 0, DD_D_WL, DD_D_WR, DD_D_GFRAC, DD_D_RSHUNT, DD_D_VPRE, DD_D_FIRST, DD_DF
};

/* What the devices of a sweep share (device pointers): the grid's layout (jaxdd's `Structure`,
 * device.py:386-575) and the flags the layers' parameters do not change. */
typedef struct dd_structure {
  int32_t np, n_layers;
  const int32_t* lid;        /* [np+2] each point's layer */
  const double* raw;         /* [np+2] unscaled spacings */
  const double* norm;        /* [n_layers] each layer's sum of raw spacings */
  const int32_t* i0;         /* [n_layers] each layer's first point */
  const int32_t* i1;         /* [n_layers] each layer's last point */
  const uint8_t* at_iface;   /* [np+2] a layer's last point before the next layer */
  const double* ifk;         /* [np+2] the interface index field of the record (dd_layout.h) */
  const double* aslot;       /* [n_layers] the layer's mobile anion slot, -1 none */
  const double* cslot;       /* [n_layers] cation slot, -1 none */
  const uint8_t* afixed;     /* [n_layers] the layer's anions are fixed */
  const uint8_t* cfixed;     /* [n_layers] */
  const int32_t* iface_row;  /* [n_layers] row of the trapped join after the layer, -1 none */
  const double* iface_kind;  /* [n_layers] that join's trap type (-1, 0, 1) */
  int32_t sfb_left, sfb_right;  /* the contact's work function is its layer's flat-band one */
  double left_elec, pre_cond, fix_ions, curr_diff, mid;
} dd_structure;

/* Build the packed record (stat, scal, iface; and y0 at each device's DD_D_FIRST voltage unless
 * NULL) of n_devices devices in lanes 0..n_devices-1 of arrays of `lane_stride` lanes. Workspace:
 * (np+2) * n_devices doubles. The record equals jaxdd_b200's host packer's for the same devices
 * but for the pairwise sums of the spacings and of the current scale (a few ulp). */
int dd_build(const dd_structure* structure, const double* layer_params,
             const double* device_params, int n_devices, int lane_stride, int k_anion,
             int k_cation, double* stat, double* scal, double* iface, double* y0,
             void* workspace, size_t workspace_bytes, void* stream);

/* ---- Transients with mobile ions (jaxdd transient.py:270-465, 537-637) -------------------- */
/* ZimT's time steps (jaxdd `TVG`, simss_input.py:155-237). Lane l's step k is at [k] (stride 0:
 * one list for every lane) or at [k * lane_stride + l] (stride = lane_stride: one per lane). The first step is at t = 0 (a steady state); a later t = 0 returns to one. */
typedef struct dd_steps {
  int32_t n_steps;
  int32_t stride;
  const double* t;             /* s */
  const double* v;             /* internal voltage, V */
  const double* g_frac;        /* generation factor */
  const int32_t* track;        /* ZimT's Track 0-3 (1 the reference state; 2 and 3 the automatic
                                  stop on five equal states in a row, `conv_var` below) */
  const int32_t* failure_mode; /* [lane_stride]: 0 stop at a failed step, 1 keep it, 2 skip it */
  int32_t zimt_sums;           /* 1: ZimT's sums in the integral current (each point's change over
                                  the interval after it); 0: over its control volume (jaxdd's) */
  int32_t zimt_ion_last;       /* 1: each species' last ion region's current alone, as ZimT 5.36
                                  has it with several regions; 0: every region's (jaxdd's) */
  /* The internal voltage an unknown of every step (jaxdd's `vint`, batch.py:552-592): 0 the
   * voltage `v` given; 1 each step's row the external current at the open circuit (`oc`),
   * else `V_int + R_series J_ext = v`. */
  int32_t vint;
  const uint8_t* oc;           /* per step, in `t`'s layout: 1 at the open circuit (`v` unread) */
  const double* r_series;      /* [lane_stride]: Ohm m^2 */
  const double* start_j_ext;   /* [lane_stride]: the external current of the start (A/m^2) */
  /* [lane_stride] each: how the automatic stop compares two states (ZimT's tolPois in V,
   * tolDens relative). NULL: no two states are equal (Track 2 and 3 never stop). */
  const double* tol_pois;
  const double* tol_dens;
  /* For ZimT's tJFile columns (dd_transient_out.columns): each lane's layers, [3][n_layers]
   * [lane_stride] (each layer's first point i0, its last i1, its thickness x[i1] - x[i0]),
   * 1 <= n_layers <= 8 (i0 = -1 past a lane's own layers: its columns there 0). */
  int32_t n_layers;
  const double* layers;
  /* [lane_stride] each: ZimT's convVar (1 the densities, 2 the currents within tol_curr or the
   * smaller errJ of the two states, 3 either, 4 both) and tolCurr (A/m^2). NULL: convVar 1. */
  const int32_t* conv_var;
  const double* tol_curr;
} dd_steps;

/* Outputs of dd_transient (device pointers). Per step and lane [n_steps][lane_stride]: J (A/m^2,
 * internal, SIMsalabim's sign), J_ext (with the shunt), converged, iterations, accepted (the
 * step is kept: ZimT's tJFile rows); per lane stop (0 through every step, 1 where ZimT's
 * automatic stop found the state static, 2 at a failed step: failureMode 0, or 2 with Track 1).
 * The last kept state: state [np_max+2][5][lane_stride] (V, ln n, ln p, ln a, ln c; the ions'
 * 0 outside their regions), logs [DD_MAXK][lane_stride]
 * (the slots' scales), f_bulk and f_iface [np_max+2][lane_stride] (the traps' occupations at
 * the points and on the intervals; either may be NULL). */
typedef struct dd_transient_out {
  double* J;
  double* J_ext;
  uint8_t* converged;
  int32_t* iterations;
  uint8_t* accepted;
  int32_t* stop;
  double* state;
  double* logs;
  double* f_bulk;
  double* f_iface;
  /* Q [lane_stride]: the integrated current sum_k J_k dt_k over the kept steps (C/m^2); dQ
   * [2][lane_stride]: its derivatives in ln N_ion (both species' totals) and ln mu_ion (both
   * species' mobilities), forward mode through every step. Both NULL: not computed. */
  double* Q;
  double* dQ;
  /* Each step's state (`profiles`, jaxdd transient.py:449-451): prof_state
   * [n_steps][np_max+2][5][lane_stride] the step's solution (contacts included, the ions' 0
   * outside their regions), prof_f_bulk and prof_f_iface [n_steps][np_max+2][lane_stride] the
   * traps' occupations at its end, prof_dti [n_steps][lane_stride]; kept or not. All NULL: none. */
  double* prof_state;
  double* prof_f_bulk;
  double* prof_f_iface;
  double* prof_dti;
  /* V_int [n_steps][lane_stride]: each step's internal voltage (the solution's with `vint`, else
   * the given one). NULL: not written. */
  double* V_int;
  /* ZimT's tJFile columns of each step (jaxdd transient.py:163-222), [n_steps][7 + 8 n_layers]
   * [lane_stride]: errJ, JminLeft, JminRight, JShunt, Jnion, Jpion, JD, then per layer (each
   * n_layers wide) QFLS, Jphoto, Jdir, JbulkElec, JbulkHoles, JintElec, JintHoles (at the
   * layer's right end), VL. NULL: none. */
  double* columns;
} dd_transient_out;

/* A state to start from instead of the steady state at the first step (jaxdd's
 * `solve_transient(..., initial=)`, transient.py:321-331): state [np_max+2][5][lane_stride]
 * (V, ln n, ln p, ln a, ln c; the interior points used, the ions' where mobile), f_bulk and
 * f_iface [np_max+2][lane_stride] the traps' occupations, scalars [4][lane_stride]: the state's
 * t, V_int, J_ext and dti. The slots' scales start at 1 and the first step's guess is the state
 * itself (no extrapolation). */
typedef struct dd_transient_init {
  const double* state;
  const double* f_bulk;
  const double* f_iface;
  const double* scalars;
} dd_transient_init;

/* Scratch bytes dd_transient needs for this batch. */
int dd_transient_workspace_bytes(const dd_batch* batch, size_t* bytes);

/* Every lane through its time steps: jaxdd's `solve_transient` (transient.py:537) with the
 * voltage given at every step. Each step is a Newton solve of implicit Euler with the mobile ions
 * as unknowns (5x5 blocks bordered by the ion slots, solver.py:1364-1475), the traps' occupations
 * carried from step to step (solver.py:594-614), the current with each density's change, the
 * ions' currents and the displacement current (batch.py:302-483), and ZimT's main loop
 * (transient.py:419-445: which steps are kept, dt from the last kept one). `tstat`
 * [np_max+2][DD_NT][lane_stride] the permittivity and the ions' mobilities at each point;
 * `start` [np_max+2][3][lane_stride] and `start_logs` [DD_MAXK][lane_stride] the steady state
 * at the first step (dd_solve_states at steps->v[0] with the generation factor
 * steps->g_frac[0] and no pre-bias), or `initial` (then start and start_logs may be NULL). opts:
 * tol, max_iter (Newton per step), bernoulli. Two threads a device (the twisted sweep and the
 * current split between them) unless the gradients (`Q`, `dQ`) or the internal voltage are
 * asked; then one. The host refuses the internal voltage an unknown with an ion region that
 * reaches a contact. */
int dd_transient(const dd_batch* batch, const double* tstat, const dd_steps* steps,
                 const double* start, const double* start_logs, const dd_transient_init* initial,
                 const dd_opts* opts, const dd_transient_out* out, void* workspace,
                 size_t workspace_bytes, void* stream);

/* One damped Newton step per lane from the state y (`[(np_max+2)][3][lane_stride]`, interior
 * nodes used) and the ion normalisations logs (`[K][lane_stride]`) at the voltage Vint
 * (`[lane_stride]`), ions scaled by `share`: jaxdd's `_newton_step` (solver.py:1563-1608),
 * batch.py:759-785. Writes the new state in place, the new logs, the step's size and the
 * current at the new state (integral or differential form, without the shunt). For checking a
 * single step against a CPU restatement; dd_solve does not call it. */
int dd_newton_step(const dd_batch* batch, double* y, double* logs, const double* vint,
                   double share, const dd_opts* opts, double* size, double* J, void* workspace,
                   size_t workspace_bytes, void* stream);

/* dd_solve without a workspace argument, for callers that cannot allocate device memory for
 * scratch: a plain C or foreign-function caller that holds the batch's buffers but has no device
 * allocator of its own, or a caller that must not call cudaMalloc/cudaFree between solves
 * (cudaFree waits for the whole device). It has no counterpart in the reference, whose solve
 * gets its scratch from XLA.
 *
 * The scratch is one fixed array of DD_NOALLOC_SCRATCH_BYTES in the library's own device memory
 * (reserved when the library's module loads on a device); nothing is allocated per call. A batch
 * whose dd_workspace_bytes exceeds it is refused with DD_ERR_SCRATCH (at 400 nodes a lane
 * stride of at most 640 with two ion slots, 544 with four); use dd_solve with a workspace for larger batches.
 * The first call on each device, with that device current, looks the array's address up
 * (cudaGetSymbolAddress) and keeps it, with the id of the device's context; a later call in
 * another context of that device (after cudaDeviceReset, say, which frees the array with the
 * module) looks it up again. Make the first call on a device, and the first after such a reset,
 * before any stream capture. DD_ERR_DEVICE if the lookup fails or the current device is not an
 * sm_100 part. All calls on a device share the one array and it keeps what
 * the last call left (the kernel writes every word before reading it, so nothing needs
 * clearing): calls whose work overlaps on the device race and give wrong results, so order them
 * on one stream or one at a time. Results are those of dd_solve on the same inputs. */
int dd_solve_noalloc(const dd_batch* batch, const dd_voltages* volts, const dd_opts* opts,
                     double* J, uint8_t* converged, int32_t* iterations, int32_t* lane_status,
                     int32_t* lane_steps, void* stream);

/* A human-readable name of a status code. */
const char* dd_status_string(int status);

/* ABI version: (major << 16) | minor. */
int dd_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* JAXDD_B200_H */
