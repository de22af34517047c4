"""Seeded synthetic devices for the benchmark workloads (SIMsalabim inputs built in memory).

There is no public dataset behind jaxdd's J-V benchmark; the workloads are stacks drawn from
fixed seeds and written as SIMsalabim setups (the reference's own input format), then built by
`build_device`:

* `pin_stack` — a p-i-n cell, HTL 20 nm / absorber 400 nm / ETL 30 nm, the HTL on the anode side
  (`leftElec = 1`), gaps 3.0 / 1.6 / 3.2 eV aligned at the absorber's bands, N_c 2.2e24 m^-3,
  eps_r 3.5 / 24 / 10, mobilities 1e-6 / 1e-4 / 1e-5 m^2/Vs, transport layers doped 1e22 m^-3
  with 'sfb' contacts, one neutral mid-gap bulk trap of 1e20 m^-3 (C 1e-14 m^3/s), k_direct
  1e-17 m^3/s, uniform generation 2.5e27 m^-3 s^-1 in the absorber, T 300 K, NP 300.
* `drawn_stack(k, rng)` — the same stack with per-device draws: absorber thickness U(300, 600)
  nm, absorber mobilities logU(1e-5, 1e-3), bulk traps logU(1e19, 1e22) at E_c + U(0.3, 0.8)
  eV, both interfaces' traps logU(1e12, 1e15) m^-2 (neutral, mid-gap), HTL N_A and ETL N_D
  logU(1e20, 1e23), absorber anions = cations logU(1e22, 1e24) with mobility 1e-12; devices of
  even index pre-biased at 1.0 V with their ions frozen, odd ones with free ions.
* the uneven workload — the same draws with a grid size NP ~ U{150..900} and a voltage count
  Nv ~ U{21..121} per device (`ragged_plan`), Nv voltages evenly over -0.2..1.3 V.
"""

from __future__ import annotations

import numpy as np

from .device import build_device
from .simss_input import setup_from_texts

__all__ = ["pin_stack", "pin_texts", "drawn_stack", "drawn_devices", "SEED_DRAWN", "V_SCAN", "ragged_plan",
           "ragged_voltages", "drawn_device"]

#: Seed of the per-device draws (the drawn J-V curves and the uneven grids).
SEED_DRAWN = 20261203
#: Seed of the mobile-ion stacks' draws (the transient and small-signal workloads).
SEED_ION_STACKS = 20261205
#: 61 voltages from -0.2 to 1.3 V.
V_SCAN = np.round(np.linspace(-0.2, 1.3, 61), 10)
#: The uneven workload's grid sizes and voltage counts: NP ~ U{150..900}, Nv ~ U{21..121}.
RAGGED_NP = (150, 900)
RAGGED_NV = (21, 121)


def _layer(**kv) -> str:
    base = dict(
        L="1e-7", eps_r="10", E_c="4.0", E_v="5.6", N_c="2.2e24", N_D="0", N_A="0",
        mu_n="1e-4", mu_p="1e-4", mobnDep="0", mobpDep="0", gamma_n="0", gamma_p="0",
        nu_int_n="1e5", nu_int_p="1e5", N_t_int="0", E_t_int="4.8", intTrapFile="none",
        intTrapType="0", C_n_int="1e-14", C_p_int="1e-14", N_anion="0", N_cation="0",
        mu_anion="0", mu_cation="0", ionsMayEnter="0", G_ehp="0", layerGen="0",
        fieldDepG="0", P0="0", a="1e-9", thermLengDist="2", k_f="1e6", k_direct="0",
        preLangevin="1", useLangevin="0", N_t_bulk="0", C_n_bulk="1e-14", C_p_bulk="1e-14",
        E_t_bulk="4.8", bulkTrapFile="none", bulkTrapType="0")
    base.update({k: str(v) for k, v in kv.items()})
    return "\n".join(f"{k} = {v}" for k, v in base.items()) + "\n"


def _setup(NP: int, pre: tuple[int, float, int] = (0, 0.0, 0)) -> str:
    pc, vpre, fix = pre
    rows = dict(
        T="300", l1="L1.txt", l2="L2.txt", l3="L3.txt", leftElec="1", W_L="sfb", W_R="sfb",
        S_n_L="-1", S_p_L="-1", S_n_R="-1", S_p_R="-1", R_shunt="-1", R_series="0",
        G_frac="1", genProfile="none", NP=str(NP), grad="4", currDiffInt="2", Vdist="1",
        preCond=str(pc), Vpre=repr(float(vpre)), fixIons=str(fix), Vscan="1", Vmin="-0.2",
        Vmax="1.3", Vstep="0.025", Vacc="0", NJV="61", untilVoc="0")
    return "\n".join(f"{k} = {v}" for k, v in rows.items()) + "\n"


def pin_stack(NP: int = 300):
    """The p-i-n cell of workload 1, built (jaxdd's graded grid)."""
    return build_device(setup_from_texts(pin_texts(NP)))


def pin_texts(NP: int = 300) -> dict[str, str]:
    """The SIMsalabim input texts of workload 1's p-i-n cell."""
    return {
        "simulation_setup.txt": _setup(NP),
        "L1.txt": _layer(L="20e-9", eps_r="3.5", E_c="2.6", E_v="5.6", mu_n="1e-6", mu_p="1e-6",
                         N_A="1e22"),
        "L2.txt": _layer(L="400e-9", eps_r="24", E_c="4.0", E_v="5.6", mu_n="1e-4", mu_p="1e-4",
                         N_t_bulk="1e20", E_t_bulk="4.8", k_direct="1e-17", G_ehp="2.5e27",
                         layerGen="1"),
        "L3.txt": _layer(L="30e-9", eps_r="10", E_c="4.0", E_v="7.2", mu_n="1e-5", mu_p="1e-5",
                         N_D="1e22"),
    }


def _logu(rng, lo, hi):
    return float(10 ** rng.uniform(np.log10(lo), np.log10(hi)))


def drawn_texts(k: int, rng: np.random.Generator, NP: int = 400) -> dict[str, str]:
    """The SIMsalabim input texts of device `k` of the drawn workload."""
    L_abs = rng.uniform(300e-9, 600e-9)
    mun, mup = _logu(rng, 1e-5, 1e-3), _logu(rng, 1e-5, 1e-3)
    Nt = _logu(rng, 1e19, 1e22)
    Et = 4.0 + rng.uniform(0.3, 0.8)
    Nti_l, Nti_r = _logu(rng, 1e12, 1e15), _logu(rng, 1e12, 1e15)
    NA, ND = _logu(rng, 1e20, 1e23), _logu(rng, 1e20, 1e23)
    Nion = _logu(rng, 1e22, 1e24)
    frozen = k % 2 == 0
    return {
        "simulation_setup.txt": _setup(NP, (1, 1.0, 1) if frozen else (0, 0.0, 0)),
        "L1.txt": _layer(L="20e-9", eps_r="3.5", E_c="2.6", E_v="5.6", mu_n="1e-6", mu_p="1e-6",
                         N_A=f"{NA:.6g}", N_t_int=f"{Nti_l:.6g}", E_t_int="4.8"),
        "L2.txt": _layer(L=f"{L_abs:.6g}", eps_r="24", E_c="4.0", E_v="5.6", mu_n=f"{mun:.6g}",
                         mu_p=f"{mup:.6g}", N_t_bulk=f"{Nt:.6g}", E_t_bulk=f"{Et:.6g}",
                         k_direct="1e-17", G_ehp="2.5e27", layerGen="1",
                         N_t_int=f"{Nti_r:.6g}", E_t_int="4.8",
                         N_anion=f"{Nion:.6g}", N_cation=f"{Nion:.6g}", mu_anion="1e-12",
                         mu_cation="1e-12", ionsMayEnter="1"),
        "L3.txt": _layer(L="30e-9", eps_r="10", E_c="4.0", E_v="7.2", mu_n="1e-5", mu_p="1e-5",
                         N_D=f"{ND:.6g}"),
    }


def drawn_stack(k: int, rng: np.random.Generator, NP: int = 400):
    return build_device(setup_from_texts(drawn_texts(k, rng, NP)))


def drawn_device(k: int, seed: int = SEED_DRAWN, NP: int | tuple[int, int] = 400):
    """Device `k` of the drawn workload (its draws depend only on the seed and `k`)."""
    rng = np.random.default_rng([seed, k])
    npk = NP if isinstance(NP, int) else int(rng.integers(NP[0], NP[1] + 1))
    return drawn_stack(k, rng, npk)


def ragged_plan(indices, seed: int = SEED_DRAWN) -> tuple[np.ndarray, np.ndarray]:
    """`(NP, Nv)` of the uneven workload's devices `indices`: the grid size is the first draw
    of the device's own stream (as `drawn_device` with `NP=RAGGED_NP` draws it), the voltage
    count a draw of a separate stream, so the device draws stay those of the fixed-size
    workload."""
    idx = np.asarray(indices, dtype=np.int64)
    NP = np.array([int(np.random.default_rng([seed, int(k)]).integers(RAGGED_NP[0],
                                                                      RAGGED_NP[1] + 1))
                   for k in idx])
    Nv = np.array([int(np.random.default_rng([seed, int(k), 3]).integers(RAGGED_NV[0],
                                                                         RAGGED_NV[1] + 1))
                   for k in idx])
    return NP, Nv


def ragged_voltages(Nv: int) -> np.ndarray:
    """`Nv` voltages evenly from -0.2 to 1.3 V."""
    return np.round(np.linspace(-0.2, 1.3, int(Nv)), 10)


def drawn_devices(n: int, seed: int = SEED_DRAWN, NP: int | tuple[int, int] = 400,
                  start: int = 0):
    """Devices `start .. start + n` of the drawn workload (each device's draws depend only on
    the seed and its index). `NP` an int, or `(lo, hi)` for a grid size drawn U{lo..hi}."""
    return [drawn_device(k, seed, NP) for k in range(start, start + n)]


def transient_devices(n: int, seed: int = SEED_ION_STACKS, NP: int = 400, start: int = 0):
    """The mobile-ion stacks: the drawn workload's devices with free mobile ions (its odd
    indices: the drawn J-V curves' distributions, ions in the absorber, no pre-bias),
    `start .. start + n` of them."""
    return [drawn_device(2 * k + 1, seed, NP) for k in range(start, start + n)]


def transient_steps(n_steps: int = 2000, V: float = 0.9):
    """The transient workload's steps: the steady state at 0 V (t = 0), then `n_steps` implicit-Euler
    steps at `V` log-spaced from 1 ns to 1 s, light on (G_frac 1), failureMode 1."""
    from .simss_input import TVG
    t = np.concatenate([[0.0], np.logspace(-9, 0, n_steps)])
    return TVG.steps(t, np.where(t > 0, V, 0.0), 1.0, 0, failure_mode=1)

