"""Write the device fixtures under tests/golden/ from the reference's own device builder.

    python tests/golden/make_golden.py /path/to/jaxdd-checkout

The reference (jaxdd) needs JAX, which is not installed where this runs; its device builder
(`jaxdd.device.build_device`, jaxdd src/jaxdd/device.py:1066-1079) computes in NumPy and only
imports `jax` at module level, through `jaxdd.statistics`. A stub `jax` module (NumPy behind
`jax.numpy`) is enough to import it. The package's `__init__` imports the solver, so the
package is mounted as a bare namespace instead.

Output: `devices.npz`, every array of every case's device for both grids, keyed
`<case>/<grid>/<field>`; the cases are the reference's own SimSS test inputs (tests/data/) that
this build supports. Inputs are copied next to the fixtures (`inputs/`), so that the tests can
rebuild the same devices without the reference.
"""

from __future__ import annotations

import shutil
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

#: The reference's SimSS and ZimT test cases inside this build's scope (Boltzmann, no surface
#: recombination, no field dependence, no trap files, no charged bulk traps).
CASES = (
    "thin_l1_light", "frozen_1e17_x1_thin_light", "steady_1e17_thin_light", "held_thin_light",
    "iface_charged_light", "iface_ions_light", "pin_iface_light", "region_etl_light",
    "region_htl_frozen_light", "two_regions_light", "frozen_thick_htl_dark", "diff_iface_light",
    "none_light", "resist_light", "logv_light",
    # ZimT 5.36 transients (with their tVG.txt and ZimT's tj.dat): electrons and holes, the
    # absorber's traps, and mobile ions over 2 x 50 ms and 2 x 5 s; a sweep to 1.2 V and back in
    # 2 x 100 ns in the integral and the differential current, charged interface traps through
    # it, steady states at t = 0; ion regions that reach a contact (a region of two layers over
    # 2 x 5 s, with the differential current over 2 x 50 ms, two regions per species)
    "zimt_photo_light", "zimt_traps_photo_light", "zimt_ions_fast_light", "zimt_ions_slow_light",
    "zimt_sweep_light", "zimt_sweep_diff_light", "zimt_iface_sweep_light", "zimt_steady_light",
    "zimt_region_slow_light", "zimt_region_diff_light", "zimt_regions2_light",
    # the internal voltage an unknown: the photovoltage at the open circuit after a light pulse,
    # a sweep through a series resistance and a shunt
    "zimt_tpv_light", "zimt_rseries_sweep_light",
    # ZimT's automatic stop on the photovoltage after a pulse (Track 2 against the steady state
    # before it, Track 3 against the step before)
    "zimt_track_tpv_light", "zimt_track_tpv3_light",
    # the sweep with each layer's voltage drop written (`specialOutput = spv`)
    "zimt_sweep_spv_light",
    # SimSS's curve at 0.1 mV steps around its open-circuit voltage
    "thin_l1_voc_light",
)


def _stub_jax() -> None:
    """Just enough of `jax` for the reference's NumPy-only modules to import."""
    jax = types.ModuleType("jax")
    jax.numpy = np
    jax.config = types.SimpleNamespace(update=lambda *a, **k: None)
    jax.nn = types.SimpleNamespace(sigmoid=lambda x: 1.0 / (1.0 + np.exp(-x)))

    def custom_jvp(f=None, **_):
        def wrap(g):
            g.defjvp = lambda rule: rule
            return g
        return wrap if f is None else wrap(f)

    jax.custom_jvp = custom_jvp
    jax.Array = np.ndarray
    sys.modules["jax"] = jax
    sys.modules["jax.numpy"] = np


def reference_device_module(checkout: Path):
    _stub_jax()
    pkg = types.ModuleType("jaxdd")
    pkg.__path__ = [str(checkout / "src" / "jaxdd")]
    sys.modules["jaxdd"] = pkg
    import jaxdd.device as device  # noqa: E402
    import jaxdd.simss_input as simss_input  # noqa: E402
    return device, simss_input


def fields(dev) -> dict[str, np.ndarray]:
    out = {}
    for name, value in vars(dev).items():
        if value is None:
            continue
        if isinstance(value, dict):
            for k, v in value.items():
                out[f"{name}.{k}"] = np.asarray(v, dtype=float)
        elif isinstance(value, (tuple, list)) and name in ("i0", "i1", "free"):
            out[name] = np.asarray(value, dtype=float)
        elif isinstance(value, str):
            continue
        else:
            out[name] = np.asarray(value, dtype=float)
    return out


def main(checkout: str) -> None:
    checkout = Path(checkout)
    device, simss_input = reference_device_module(checkout)
    data = checkout / "tests" / "data"
    inputs = HERE / "inputs"
    arrays = {}
    for case in CASES:
        src = data / case
        dst = inputs / case
        dst.mkdir(parents=True, exist_ok=True)
        for f in src.iterdir():
            if f.suffix in (".txt", ".dat"):
                shutil.copyfile(f, dst / f.name)
        setup = simss_input.read_setup(src / "simulation_setup.txt")
        for grid in ("simss", "graded"):
            dev = device.build_device(setup, grid=grid)
            for k, v in fields(dev).items():
                arrays[f"{case}/{grid}/{k}"] = v
    np.savez_compressed(HERE / "devices.npz", **arrays)
    print(f"{len(CASES)} cases, {len(arrays)} arrays -> {HERE / 'devices.npz'}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
