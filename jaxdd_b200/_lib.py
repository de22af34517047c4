"""ctypes binding of the C ABI in include/jaxdd_b200.h (the library built by jaxdd_b200.build).

Loading fails loudly when the library is missing: the package has no other compute path.
"""

from __future__ import annotations

import ctypes
from functools import lru_cache

from .build import LIB

#: field counts of jaxdd_b200/csrc/dd_layout.h
DD_NF = 26
DD_NS_BASE = 20
DD_NIF = 10
DD_MAXIF = 4
DD_MAXK = 4
DD_NBUF = 4

S = {name: k for k, name in enumerate((
    "OFFN", "OFFP", "MUN", "MUP", "H", "DX", "FACL", "FACM", "FACU", "FAC", "SP", "SC", "DOP",
    "KD", "NI2", "NT", "CNT", "CPT", "NT0", "PT0", "G", "ASLOT", "CSLOT", "AFIX", "CFIX", "IFK"))}
C = {name: k for k, name in enumerate((
    "VT", "L", "V0", "VL", "LEFT", "LNNL", "LNPL", "LNNR", "LNPR", "JSCALE", "GSHUNT",
    "PRECOND", "VPRE", "FIXIONS", "GFRAC", "NFLOOR", "NP", "CURRDIFF", "HSUM", "MID"))}
I = {name: k for k, name in enumerate((
    "NT", "CN", "CP", "NT0LO", "PT0LO", "NT0HI", "PT0HI", "IW", "CHARGE", "CWE"))}
assert len(S) == DD_NF and len(C) == DD_NS_BASE and len(I) == DD_NIF

DD_MODE_BATCH, DD_MODE_JV = 0, 1
DD_BERNOULLI = {"exact": 0, "simss": 1}
DD_PRECISION = {"fp64": 0, "mixed": 1}
DD_LANE_PREBIAS_FAILED = 1

#: every symbol include/jaxdd_b200.h declares
EXPORTS = ("dd_abi_version", "dd_status_string", "dd_workspace_bytes", "dd_solve", "dd_tune",
           "dd_newton_step", "dd_solve_noalloc", "dd_solve_states", "dd_adjoint_workspace_bytes",
           "dd_adjoint", "dd_observables", "dd_admittance_workspace_bytes", "dd_admittance",
           "dd_build", "dd_transient_workspace_bytes", "dd_transient",
           "dd_admittance_ions_workspace_bytes", "dd_admittance_ions")

#: the transient's per-point record fields (include/jaxdd_b200.h DD_NT)
DD_NT = 3
#: the tJFile columns: the scalar ones, then 8 per layer, at most this many layers
DD_COL_SCALARS, DD_COL_MAXL = 7, 8
COL_SCALARS = ("errJ", "JminLeft", "JminRight", "JShunt", "Jnion", "Jpion", "JD")
COL_LAYER = ("QFLS", "Jphoto", "Jdir", "JbulkElec", "JbulkHoles", "JintElec", "JintHoles", "VL")

#: include/jaxdd_b200.h's per-layer and per-device parameter fields of dd_build
LAYER_FIELDS = ("L", "eps_r", "E_c", "E_v", "N_c", "N_D", "N_A", "mu_n", "mu_p", "k_direct",
                "N_t_bulk", "E_t_bulk", "C_n_bulk", "C_p_bulk", "nu_int_n", "nu_int_p",
                "N_t_int", "E_t_int", "C_n_int", "C_p_int", "G_ehp", "N_anion", "N_cation")
DEVICE_FIELDS = ("T", "W_L", "W_R", "G_frac", "R_shunt", "Vpre", "first")
DD_MAXLAYERS = 16

#: dd_solve_noalloc's fixed scratch (include/jaxdd_b200.h DD_NOALLOC_SCRATCH_BYTES)
DD_NOALLOC_SCRATCH_BYTES = 64 << 20
DD_ERR_SCRATCH = 5
#: include/jaxdd_b200.h DD_SOLVE_FORMS: the solve's launch forms (block, work queue)
DD_SOLVE_FORMS = 4
SOLVE_FORMS = ({"block": 32, "queue": True}, {"block": 64, "queue": True},
               {"block": 32, "queue": False}, {"block": 64, "queue": False})


class DdBatch(ctypes.Structure):
    _fields_ = [("n_lanes", ctypes.c_int32), ("lane_stride", ctypes.c_int32),
                ("np_max", ctypes.c_int32), ("k_anion", ctypes.c_int32),
                ("k_cation", ctypes.c_int32), ("stat", ctypes.c_void_p),
                ("scal", ctypes.c_void_p), ("iface", ctypes.c_void_p), ("y0", ctypes.c_void_p)]


class DdVoltages(ctypes.Structure):
    _fields_ = [("v", ctypes.c_void_p), ("offset", ctypes.c_void_p), ("count", ctypes.c_void_p)]


class DdStructure(ctypes.Structure):
    _fields_ = [("np", ctypes.c_int32), ("n_layers", ctypes.c_int32)] + [
        (name, ctypes.c_void_p) for name in ("lid", "raw", "norm", "i0", "i1", "at_iface", "ifk",
                                             "aslot", "cslot", "afixed", "cfixed", "iface_row",
                                             "iface_kind")] + [
        ("sfb_left", ctypes.c_int32), ("sfb_right", ctypes.c_int32),
        ("left_elec", ctypes.c_double), ("pre_cond", ctypes.c_double),
        ("fix_ions", ctypes.c_double), ("curr_diff", ctypes.c_double), ("mid", ctypes.c_double)]


class DdSteps(ctypes.Structure):
    _fields_ = [("n_steps", ctypes.c_int32), ("stride", ctypes.c_int32), ("t", ctypes.c_void_p),
                ("v", ctypes.c_void_p), ("g_frac", ctypes.c_void_p), ("track", ctypes.c_void_p),
                ("failure_mode", ctypes.c_void_p), ("zimt_sums", ctypes.c_int32),
                ("zimt_ion_last", ctypes.c_int32), ("vint", ctypes.c_int32),
                ("oc", ctypes.c_void_p), ("r_series", ctypes.c_void_p),
                ("start_j_ext", ctypes.c_void_p), ("tol_pois", ctypes.c_void_p),
                ("tol_dens", ctypes.c_void_p), ("n_layers", ctypes.c_int32),
                ("layers", ctypes.c_void_p), ("conv_var", ctypes.c_void_p),
                ("tol_curr", ctypes.c_void_p)]


class DdTransientOut(ctypes.Structure):
    _fields_ = [(name, ctypes.c_void_p) for name in (
        "J", "J_ext", "converged", "iterations", "accepted", "stop", "state", "logs", "f_bulk",
        "f_iface", "Q", "dQ", "prof_state", "prof_f_bulk", "prof_f_iface", "prof_dti", "V_int",
        "columns")]


class DdTransientInit(ctypes.Structure):
    _fields_ = [(name, ctypes.c_void_p) for name in ("state", "f_bulk", "f_iface", "scalars")]


class DdOpts(ctypes.Structure):
    _fields_ = [("tol", ctypes.c_double), ("max_iter", ctypes.c_int32),
                ("start_iter", ctypes.c_int32), ("strict", ctypes.c_int32),
                ("bernoulli", ctypes.c_int32), ("mode", ctypes.c_int32),
                ("precision", ctypes.c_int32), ("reserved", ctypes.c_int32)]


@lru_cache(maxsize=1)
def lib() -> ctypes.CDLL:
    if not LIB.exists():
        raise RuntimeError(f"the jaxdd_b200 CUDA library is not built ({LIB}); run "
                           "`python -m jaxdd_b200.build` (or __graft_entry__.build())")
    so = ctypes.CDLL(str(LIB))
    p = ctypes.c_void_p
    so.dd_abi_version.restype = ctypes.c_int
    so.dd_status_string.restype = ctypes.c_char_p
    so.dd_status_string.argtypes = [ctypes.c_int]
    so.dd_workspace_bytes.restype = ctypes.c_int
    so.dd_workspace_bytes.argtypes = [ctypes.POINTER(DdBatch), ctypes.POINTER(ctypes.c_size_t)]
    so.dd_solve.restype = ctypes.c_int
    so.dd_solve.argtypes = [ctypes.POINTER(DdBatch), ctypes.POINTER(DdVoltages),
                            ctypes.POINTER(DdOpts), p, p, p, p, p, p, ctypes.c_size_t, p]
    so.dd_tune.restype = ctypes.c_int
    so.dd_tune.argtypes = [ctypes.POINTER(DdBatch), ctypes.POINTER(DdVoltages),
                           ctypes.POINTER(DdOpts), p, p, p, p, p, p, ctypes.c_size_t, p, p, p]
    so.dd_newton_step.restype = ctypes.c_int
    so.dd_newton_step.argtypes = [ctypes.POINTER(DdBatch), p, p, p, ctypes.c_double,
                                  ctypes.POINTER(DdOpts), p, p, p, ctypes.c_size_t, p]
    so.dd_solve_states.restype = ctypes.c_int
    so.dd_solve_states.argtypes = [ctypes.POINTER(DdBatch), ctypes.POINTER(DdVoltages),
                                   ctypes.POINTER(DdOpts), p, p, p, p, p, p, p, p, p,
                                   ctypes.c_int, p, ctypes.c_size_t, p]
    so.dd_adjoint_workspace_bytes.restype = ctypes.c_int
    so.dd_adjoint_workspace_bytes.argtypes = [ctypes.POINTER(DdBatch),
                                              ctypes.POINTER(ctypes.c_size_t)]
    so.dd_adjoint.restype = ctypes.c_int
    so.dd_adjoint.argtypes = [ctypes.POINTER(DdBatch), ctypes.POINTER(DdVoltages),
                              ctypes.POINTER(DdOpts), p, p, p, p, p, p, ctypes.c_int, p, p, p, p,
                              ctypes.c_size_t, p]
    so.dd_observables.restype = ctypes.c_int
    so.dd_observables.argtypes = [ctypes.POINTER(DdBatch), ctypes.POINTER(DdVoltages), p, p, p,
                                  p, ctypes.c_int, p, p, p, p, p, p, p, p, p]
    so.dd_admittance_workspace_bytes.restype = ctypes.c_int
    so.dd_admittance_workspace_bytes.argtypes = [ctypes.POINTER(DdBatch), ctypes.c_int,
                                                 ctypes.POINTER(ctypes.c_size_t)]
    so.dd_admittance.restype = ctypes.c_int
    so.dd_admittance.argtypes = [ctypes.POINTER(DdBatch), p, p, p, p, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_double, p, p, ctypes.c_size_t, p]
    so.dd_build.restype = ctypes.c_int
    so.dd_build.argtypes = [ctypes.POINTER(DdStructure), p, p, ctypes.c_int, ctypes.c_int,
                            ctypes.c_int, ctypes.c_int, p, p, p, p, p, ctypes.c_size_t, p]
    so.dd_admittance_ions_workspace_bytes.restype = ctypes.c_int
    so.dd_admittance_ions_workspace_bytes.argtypes = [ctypes.POINTER(DdBatch), ctypes.c_int,
                                                      ctypes.POINTER(ctypes.c_size_t)]
    so.dd_admittance_ions.restype = ctypes.c_int
    so.dd_admittance_ions.argtypes = [ctypes.POINTER(DdBatch), p, p, p, p, p, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_double, p, p, ctypes.c_size_t, p]
    so.dd_transient_workspace_bytes.restype = ctypes.c_int
    so.dd_transient_workspace_bytes.argtypes = [ctypes.POINTER(DdBatch),
                                                ctypes.POINTER(ctypes.c_size_t)]
    so.dd_transient.restype = ctypes.c_int
    so.dd_transient.argtypes = [ctypes.POINTER(DdBatch), p, ctypes.POINTER(DdSteps), p, p,
                                ctypes.POINTER(DdTransientInit), ctypes.POINTER(DdOpts),
                                ctypes.POINTER(DdTransientOut), p, ctypes.c_size_t, p]
    so.dd_solve_noalloc.restype = ctypes.c_int
    so.dd_solve_noalloc.argtypes = [ctypes.POINTER(DdBatch), ctypes.POINTER(DdVoltages),
                                    ctypes.POINTER(DdOpts), p, p, p, p, p, p]
    return so


def check(status: int, what: str) -> None:
    if status != 0:
        raise RuntimeError(f"{what}: {lib().dd_status_string(status).decode()} ({status})")
