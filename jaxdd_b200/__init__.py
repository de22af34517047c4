"""jaxdd_b200: jaxdd's batched steady-state drift-diffusion J-V solve, B200-native.

The drop-in API of jaxdd (`build_device`, `prepare`, `solve_jv`, `solve_batch`, jaxdd
src/jaxdd/__init__.py:14-29), `solve_state` and `solve_states`, `solve_transient` (ZimT's time
steps with mobile ions) and its `tj_columns`, `solve_impedance`, plus `solve_uneven` (every
device its own grid size and voltage list, in one launch), over hand-written sm_100a CUDA
kernels behind a C ABI (include/jaxdd_b200.h). Device building is host NumPy, as in jaxdd; the
solve runs only on the GPU (no CPU fallback: without the built library the solvers raise).
"""

from .batch import (Batch, external_voltages, prepare, solve_batch, solve_states,
                    solve_uneven, tune)
from .device import Device, build_device, layer_points, make_grid
from .impedance import ImpedanceResult, solve_impedance
from .simss_input import (TVG, Layer, Setup, check_supported, read_setup, read_tvg,
                          setup_from_texts, simss_voltages)
from .solver import JVResult, StateResult, solve_jv, solve_state
from .transient import TransientResult, TransientState, solve_transient, tj_columns

__version__ = "0.1.0"

__all__ = [
    "Batch", "Device", "ImpedanceResult", "JVResult", "Layer", "Setup", "StateResult", "TVG",
    "TransientResult", "TransientState", "build_device", "check_supported", "external_voltages",
    "layer_points", "make_grid", "prepare", "read_setup", "read_tvg", "setup_from_texts",
    "simss_voltages", "solve_batch", "solve_impedance", "solve_jv", "solve_state", "solve_states",
    "solve_transient", "solve_uneven", "tj_columns", "tune",
]
