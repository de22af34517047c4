"""The C ABI without a GPU: the library builds for sm_100a, loads, and exports every symbol the
header declares; the packer writes the layout the kernel reads."""

import re
from pathlib import Path

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from jaxdd_b200 import _lib
from jaxdd_b200.batch import prepare
from jaxdd_b200.device import build_device
from jaxdd_b200.simss_input import read_setup


def test_library_exports_every_declared_symbol():
    header = (ROOT / "include" / "jaxdd_b200.h").read_text()
    declared = set(re.findall(r"^\s*(?:int|const char\*)\s+(dd_\w+)\(", header, re.M))
    assert declared == set(_lib.EXPORTS)
    so = _lib.lib()
    for name in declared:
        assert hasattr(so, name), name
    assert so.dd_abi_version() >> 16 == 1
    assert so.dd_status_string(0).decode() == "ok"


def test_layout_constants_match_the_header():
    text = (ROOT / "jaxdd_b200" / "csrc" / "dd_layout.h").read_text()
    start = text.index("enum StaticField")
    body = text[start:text.index("DD_NF", start)]
    names = re.findall(r"\bS_(\w+)", body)
    assert names == list(_lib.S)
    assert f"DD_MAXIF = {_lib.DD_MAXIF}" in text and f"DD_MAXK = {_lib.DD_MAXK}" in text


def test_workspace_query_and_argument_checks():
    dev = build_device(read_setup(GOLDEN / "inputs" / "thin_l1_light" / "simulation_setup.txt"))
    b = prepare([dev])
    desc = _lib.DdBatch(b["n"], b["Bp"], b["np_max"], b["ka"], b["kc"], 1, 1, 1, 1)
    import ctypes
    size = ctypes.c_size_t(0)
    assert _lib.lib().dd_workspace_bytes(ctypes.byref(desc), ctypes.byref(size)) == 0
    nodes = b["np_max"] + 2
    # four state buffers, the frozen ions, the sweep's c'/d' (two slots), the queue's counter
    assert size.value == 8 * nodes * b["Bp"] * (4 * 3 + 2 + 12 + 3 * 2) + 256
    bad = _lib.DdBatch(b["n"], 31, b["np_max"], 1, 1, 1, 1, 1, 1)
    assert _lib.lib().dd_workspace_bytes(ctypes.byref(bad), ctypes.byref(size)) == 1


def test_the_fixed_scratch_solve_refuses_a_batch_larger_than_its_array():
    """dd_solve_noalloc checks the batch's scratch against its fixed array before any CUDA call:
    at 400 nodes and two ion slots a lane stride of 640 fits, 672 does not."""
    import ctypes
    size = ctypes.c_size_t(0)
    fits = _lib.DdBatch(640, 640, 400, 1, 1, 1, 1, 1, 1)
    over = _lib.DdBatch(672, 672, 400, 1, 1, 1, 1, 1, 1)
    so = _lib.lib()
    assert so.dd_workspace_bytes(ctypes.byref(fits), ctypes.byref(size)) == 0
    assert size.value <= _lib.DD_NOALLOC_SCRATCH_BYTES
    assert so.dd_workspace_bytes(ctypes.byref(over), ctypes.byref(size)) == 0
    assert size.value > _lib.DD_NOALLOC_SCRATCH_BYTES
    v = _lib.DdVoltages(1, 1, 1)
    opts = _lib.DdOpts(1e-10, 60, 60, 0, 0, 0, 0, 0)
    st = so.dd_solve_noalloc(ctypes.byref(over), ctypes.byref(v), ctypes.byref(opts),
                             1, 1, 1, 1, None, None)
    assert st == _lib.DD_ERR_SCRATCH
    assert "scratch" in so.dd_status_string(st).decode()
    text = (ROOT / "include" / "jaxdd_b200.h").read_text()
    assert f"DD_ERR_SCRATCH {_lib.DD_ERR_SCRATCH}" in text
    assert "DD_NOALLOC_SCRATCH_BYTES (64u << 20)" in text


def test_packer_writes_the_stencils():
    dev = build_device(read_setup(GOLDEN / "inputs" / "two_regions_light" / "simulation_setup.txt"))
    b = prepare([dev])
    S = _lib.S
    col = b["stat"][:, :, 0]
    NP = len(dev.x) - 2
    assert np.array_equal(col[:NP + 2, S["OFFN"]], dev.offset_n)
    assert b["ka"] == 2 and b["kc"] == 2
    assert set(np.unique(col[:NP + 2, S["ASLOT"]])) == {-1.0, 0.0, 1.0}
    assert np.sum(col[:, S["IFK"]] >= 0) == 2  # two trapped interfaces
    assert b["scal"][_lib.DD_NS_BASE:_lib.DD_NS_BASE + 4, 0].min() > 0


def test_mixed_grid_sizes_are_refused_unless_ragged():
    a = build_device(read_setup(GOLDEN / "inputs" / "thin_l1_light" / "simulation_setup.txt"))
    from jaxdd_b200.workloads import pin_stack
    c = pin_stack(NP=120)
    with pytest.raises(ValueError, match="one grid size"):
        prepare([a, c])
    b = prepare([a, c], ragged=True)
    assert b["np_max"] == 400 and list(b["NP"]) == [400, 120]


def test_uneven_plan_and_padded_concat():
    """The uneven workload's grid sizes and voltage counts stay in range and repeat; parts of
    different grid sizes concatenate with the smaller ones padded by empty nodes, their own
    records unchanged."""
    from jaxdd_b200.batch import concat, solve_uneven
    from jaxdd_b200.workloads import RAGGED_NP, drawn_device, ragged_plan, ragged_voltages
    NPs, nv = ragged_plan(range(200))
    assert NPs.min() >= 150 and NPs.max() <= 900 and nv.min() >= 21 and nv.max() <= 121
    assert np.array_equal(ragged_plan([7, 3])[0], NPs[[7, 3]])
    assert len(drawn_device(7, NP=RAGGED_NP).x) == NPs[7] + 2
    V = ragged_voltages(21)
    assert len(V) == 21 and V[0] == -0.2 and V[-1] == 1.3
    small = prepare([drawn_device(k, NP=(150, 160)) for k in range(32)], ragged=True)
    large = prepare([drawn_device(k, NP=(300, 310)) for k in range(32, 64)], ragged=True)
    with pytest.raises(ValueError):
        concat([small, large])
    both = concat([small, large], ragged=True)
    assert both["np_max"] == large["np_max"] and both["Bp"] == 64
    n = small["np_max"] + 2
    assert np.array_equal(both["stat"][:n, :, :32], small["stat"])
    assert np.all(both["stat"][n:, _lib.S["IFK"], :32] == -2.0)
    assert np.all(both["stat"][n:, _lib.S["SP"], :32] == 1.0)
    assert np.array_equal(both["stat"][:, :, 32:], large["stat"])
    assert np.array_equal(both["lane_of"][32:], large["lane_of"] + 32)
    with pytest.raises(ValueError):
        solve_uneven(small, [V] * 31)
    with pytest.raises(ValueError):
        solve_uneven(small, [V] * 31 + [[]])


def test_the_header_compiles_as_c():
    """The C ABI's header is plain C99: a C, cgo or FFI caller can include it."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    r = subprocess.run([gcc, "-x", "c", "-std=c99", "-Wall", "-Werror", "-fsyntax-only",
                        str(ROOT / "include" / "jaxdd_b200.h")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_the_transient_refuses_inconsistent_arguments_before_any_launch():
    """`dd_transient`'s checks, which return before any CUDA call: a start or a given state
    half given, profiles half asked, the internal voltage an unknown without its steps' data,
    columns without layers, and a workspace below its query. The pointers
    are placeholders the checks never read through."""
    import ctypes
    so = _lib.lib()
    desc = _lib.DdBatch(32, 32, 100, 1, 1, 1, 1, 1, 1)
    size = ctypes.c_size_t(0)
    assert so.dd_transient_workspace_bytes(ctypes.byref(desc), ctypes.byref(size)) == 0
    ws = size.value
    opts = _lib.DdOpts(1e-10, 60, 60, 0, 0, 0, 0, 0)

    def steps(**kw):
        base = dict(n_steps=4, stride=0, t=1, v=1, g_frac=1, track=1, failure_mode=1)
        base.update(kw)
        return _lib.DdSteps(**base)

    def out(**kw):
        base = {k: 1 for k in ("J", "J_ext", "converged", "iterations", "accepted", "stop",
                               "state", "logs")}
        base.update(kw)
        return _lib.DdTransientOut(**base)

    def call(st=None, o=None, start=1, logs=1, init=None, bytes_=ws):
        return so.dd_transient(ctypes.byref(desc), 1, ctypes.byref(st or steps()), start, logs,
                               init, ctypes.byref(opts), ctypes.byref(o or out()), 1, bytes_,
                               None)

    ARGS, WORKSPACE = 1, 2
    assert call(start=None) == ARGS  # no start and no given state
    half = _lib.DdTransientInit(1, 1, None, 1)
    assert call(init=ctypes.byref(half)) == ARGS
    assert call(o=out(prof_state=1, prof_f_bulk=1)) == ARGS  # profiles half asked
    assert call(st=steps(vint=1)) == ARGS  # the internal voltage without its steps' data
    assert call(st=steps(stride=7)) == ARGS
    assert call(o=out(columns=1)) == ARGS  # columns without layers
    assert call(st=steps(n_layers=9, layers=1), o=out(columns=1)) == ARGS  # too many layers
    assert call(bytes_=ws - 1) == WORKSPACE


def test_the_solvers_refuse_without_a_gpu():
    """No CPU fallback: without a CUDA GPU the one-device solvers raise before any solve."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from jaxdd_b200 import solve_jv, solve_state
    dev = build_device(read_setup(GOLDEN / "inputs" / "thin_l1_light" / "simulation_setup.txt"))
    with pytest.raises(RuntimeError, match="needs a CUDA GPU"):
        solve_state(dev, 0.0)
    with pytest.raises(RuntimeError, match="needs a CUDA GPU"):
        solve_jv(dev, [0.0, 0.5])


def test_the_public_names_are_the_references_in_scope():
    """The names jaxdd exports (src/jaxdd/__init__.py) that lie on the path are exported here
    under the same names; `solve_impedance` checks `ion_flux` as jaxdd does before any solve."""
    import jaxdd_b200
    for name in ("TVG", "Device", "ImpedanceResult", "JVResult", "Layer", "Setup",
                 "StateResult", "TransientResult", "TransientState", "build_device",
                 "check_supported", "external_voltages", "prepare", "read_setup", "read_tvg",
                 "setup_from_texts", "simss_voltages", "solve_batch", "solve_impedance",
                 "solve_jv", "solve_state", "solve_states", "solve_transient", "tj_columns"):
        assert name in jaxdd_b200.__all__ and hasattr(jaxdd_b200, name), name
    dev = build_device(read_setup(GOLDEN / "inputs" / "thin_l1_light" / "simulation_setup.txt"))
    with pytest.raises(ValueError, match="ion_flux"):
        jaxdd_b200.solve_impedance(prepare([dev]), [1e3], ion_flux="sites")
