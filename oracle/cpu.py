"""TEST INFRASTRUCTURE ONLY — the C++ restatement of the oracle's `solve_batch` (oracle/dd_cpu.cpp).

`solve_batch` here takes the tree `oracle.dd.prepare` builds and solves its devices one at a
time in compiled, single-threaded FP64 code: jaxdd's batched J-V solve (src/jaxdd/batch.py:
1136-1208) as a CPU implementation runs it. It serves as the timed CPU baseline (one process per
host core, jaxdd benchmarks/run.py:18-26's protocol) and as a fast second checker; it is pinned to
`oracle.dd.solve_batch` by tests/test_oracle_cpu.py. The product never imports it.

`build()` compiles oracle/dd_cpu.cpp with g++ into oracle/lib/libddcpu.so (generic x86-64 code,
so that the library built here runs on any host it travels to).
"""

from __future__ import annotations

import ctypes
import subprocess
from functools import lru_cache
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "dd_cpu.cpp"
LIB = HERE / "lib" / "libddcpu.so"
FLAGS = ["-O3", "-std=c++17", "-fPIC", "-shared", "-fno-fast-math"]

_D = ctypes.POINTER(ctypes.c_double)
_ARRAYS = ("fac_l", "fac_m", "fac_u", "fac", "sP", "sC", "dop", "a_mask", "c_mask", "a_fix",
           "c_fix", "x", "h", "N_c", "ni", "E_c", "offset_n", "offset_p", "mu_n", "mu_p", "G",
           "kd", "ni2", "Nt", "Cn", "Cp", "nt0", "pt0", "ti")
_SCALARS = ("Vt", "g_frac", "L", "V0", "VL", "W_L", "W_R", "ln_n_left", "ln_n_right",
            "ln_p_left", "ln_p_right", "J_scale", "left_elec", "G_shunt", "pre_cond", "V_pre",
            "fix_ions", "curr_diff", "n_floor")


class DdcDevice(ctypes.Structure):
    _fields_ = ([("NP", ctypes.c_int32), ("ka", ctypes.c_int32), ("kc", ctypes.c_int32),
                 ("pad", ctypes.c_int32)]
                + [(k, _D) for k in _ARRAYS[:-1]]
                + [("ti", _D), ("iface", ctypes.POINTER(ctypes.c_uint8)), ("hL", _D),
                   ("a_slots", _D), ("c_slots", _D), ("a_totals", _D), ("c_totals", _D)]
                + [(k, ctypes.c_double) for k in _SCALARS])


def build(force: bool = False) -> Path:
    """Compile the restatement if its source is newer than the library."""
    LIB.parent.mkdir(exist_ok=True)
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    proc = subprocess.run(["g++", *FLAGS, "-o", str(tmp), str(SRC)], capture_output=True,
                          text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"g++ failed on {SRC.name}:\n{proc.stderr}")
    tmp.replace(LIB)
    return LIB


@lru_cache(maxsize=1)
def lib() -> ctypes.CDLL:
    so = ctypes.CDLL(str(build()))
    so.ddc_solve_batch.restype = ctypes.c_int
    so.ddc_solve_batch.argtypes = [ctypes.POINTER(DdcDevice), _D, ctypes.c_int, ctypes.c_double,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, _D,
                                   ctypes.POINTER(ctypes.c_uint8),
                                   ctypes.POINTER(ctypes.c_int32)]
    return so


def _arr(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


def device(tree: dict, b: int) -> tuple[DdcDevice, list]:
    """Device `b` of an `oracle.dd.prepare` tree as the C struct (and the arrays it points into,
    which must outlive it)."""
    s, ion, rec = tree["s"], tree["ion"], tree["rec"]
    keep: list = []

    def ptr(a, dtype=np.float64, ctype=_D):
        a = _arr(a, dtype)
        keep.append(a)
        return a.ctypes.data_as(ctype)

    NP = tree["x"].shape[1] - 2
    ti = np.stack([tree["ti"][k][b] for k in ("Nt", "Cn", "Cp", "nt0_lo", "pt0_lo", "nt0_hi",
                                              "pt0_hi", "iw", "charge", "cwe")])
    src = {"fac_l": s["fac_l"][b], "fac_m": s["fac_m"][b], "fac_u": s["fac_u"][b],
           "fac": s["fac"][b], "sP": s["sP"][b], "sC": s["sC"][b], "dop": s["dop"][b],
           "a_mask": s["a_mask"][b], "c_mask": s["c_mask"][b], "a_fix": s["a_fix"][b],
           "c_fix": s["c_fix"][b], "x": tree["x"][b], "h": tree["h"][b], "N_c": tree["N_c"][b],
           "ni": tree["ni"][b], "E_c": tree["E_c"][b], "offset_n": tree["offset_n"][b],
           "offset_p": tree["offset_p"][b], "mu_n": tree["mu_n"][b], "mu_p": tree["mu_p"][b],
           "G": tree["G"][b], "kd": rec["kd"][b], "ni2": rec["ni2"][b], "Nt": rec["Nt"][b],
           "Cn": rec["Cn"][b], "Cp": rec["Cp"][b], "nt0": rec["nt0"][b], "pt0": rec["pt0"][b],
           "ti": ti}
    d = DdcDevice()
    d.NP = NP
    d.ka = ion["a_slots"].shape[1]
    d.kc = ion["c_slots"].shape[1]
    for k in _ARRAYS:
        setattr(d, k, ptr(src[k]))
    d.iface = ptr(tree["iface"][b], np.uint8, ctypes.POINTER(ctypes.c_uint8))
    d.hL = ptr(ion["hL"][b])
    d.a_slots = ptr(ion["a_slots"][b])
    d.c_slots = ptr(ion["c_slots"][b])
    d.a_totals = ptr(ion["a_totals"][b])
    d.c_totals = ptr(ion["c_totals"][b])
    vals = {"Vt": tree["Vt"][b], "g_frac": tree["g_frac"][b], "L": tree["L"][b],
            "V0": tree["V0"][b], "VL": tree["VL"][b], "W_L": tree["W_L"][b],
            "W_R": tree["W_R"][b], "ln_n_left": tree["ln_n_left"][b],
            "ln_n_right": tree["ln_n_right"][b], "ln_p_left": tree["ln_p_left"][b],
            "ln_p_right": tree["ln_p_right"][b], "J_scale": tree["J_scale"][b],
            "left_elec": tree["left_elec"][b], "G_shunt": tree["G_shunt"][b],
            "pre_cond": tree["pre_cond"][b], "V_pre": tree["V_pre"][b],
            "fix_ions": tree["fix_ions"][b], "curr_diff": tree["curr_diff"][b],
            "n_floor": s["n_floor"][b][0]}
    for k in _SCALARS:
        setattr(d, k, float(vals[k]))
    return d, keep


def solve_batch(tree: dict, voltages, tol: float = 1e-10, max_iter: int = 60,
                first_max_iter: int = 6, bernoulli_name: str = "exact"):
    """`oracle.dd.solve_batch` in compiled code: `(J, converged, iterations)`, devices x
    voltages in the caller's order, the shunt's current added."""
    V = _arr(voltages)
    nb = tree["x"].shape[0]
    J = np.zeros((nb, V.size))
    ok = np.zeros((nb, V.size), dtype=np.uint8)
    its = np.zeros((nb, V.size), dtype=np.int32)
    so = lib()
    for b in range(nb):
        d, keep = device(tree, b)
        st = so.ddc_solve_batch(ctypes.byref(d), V.ctypes.data_as(_D), V.size, tol, max_iter,
                                first_max_iter, 1 if bernoulli_name == "simss" else 0,
                                J[b].ctypes.data_as(_D),
                                ok[b].ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                                its[b].ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
        if st != 0:
            raise ValueError(f"ddc_solve_batch refused device {b} ({st})")
        del keep
    return J, ok.astype(bool), its


def solve_batch_mixed(tree: dict, voltages, theta: float, tol: float = 1e-10,
                      max_iter: int = 60, bernoulli_name: str = "exact"):
    """`solve_batch` (one pass at `max_iter`) with the per-lane mixed-precision sweep of
    oracle/dd_cpu.cpp: an FP32 block sweep (each node's rows and unknowns scaled by its diagonal
    block) while the lane's last Newton step exceeds `theta`, FP64 after. Returns `(J,
    converged, iterations, stats)`, stats per device: steps with an FP32 sweep, steps with an
    FP64 one, the geometric mean of the step-size ratio after an FP32 step, how many ratios."""
    so = lib()
    if not hasattr(so, "_mixed_bound"):
        so.ddc_solve_batch_mixed.restype = ctypes.c_int
        so.ddc_solve_batch_mixed.argtypes = [
            ctypes.POINTER(DdcDevice), _D, ctypes.c_int, ctypes.c_double, ctypes.c_int,
            ctypes.c_int, ctypes.c_double, _D, ctypes.POINTER(ctypes.c_uint8),
            ctypes.POINTER(ctypes.c_int32), _D]
        so._mixed_bound = True
    V = _arr(voltages)
    nb = tree["x"].shape[0]
    J = np.zeros((nb, V.size))
    ok = np.zeros((nb, V.size), dtype=np.uint8)
    its = np.zeros((nb, V.size), dtype=np.int32)
    stats = np.zeros((nb, 4))
    for b in range(nb):
        d, keep = device(tree, b)
        st = so.ddc_solve_batch_mixed(
            ctypes.byref(d), V.ctypes.data_as(_D), V.size, tol, max_iter,
            1 if bernoulli_name == "simss" else 0, float(theta), J[b].ctypes.data_as(_D),
            ok[b].ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
            its[b].ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), stats[b].ctypes.data_as(_D))
        if st != 0:
            raise ValueError(f"ddc_solve_batch_mixed refused device {b} ({st})")
        del keep
    return J, ok.astype(bool), its, stats
