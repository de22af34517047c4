"""SIMsalabim input files: `simulation_setup.txt`, the layer files it names and ZimT's `tVGFile`.

The file format is SIMsalabim's: each line `name = value`, `*` starting a comment anywhere on
the line, names in any order (a later one replaces an earlier one). Each line is read by one
regular expression. Values stay strings until a consumer converts them, so that an unsupported
parameter can be refused by name (`check_supported`). The errors the checks raise carry SimSS's
and ZimT's own messages word for word, since callers (and jaxdd's tests) match them; the
public names and signatures are those of jaxdd's reader (jaxdd src/jaxdd/simss_input.py).
"""

from __future__ import annotations

import io
import itertools
import os
import re
from collections.abc import Callable, Iterator, Mapping
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

__all__ = [
    "Layer",
    "Setup",
    "TVG",
    "check_supported",
    "ion_region_problems",
    "ion_regions",
    "parse_parameters",
    "read_setup",
    "read_tvg",
    "setup_from_texts",
    "simss_voltages",
]

# `name = value` once the comment is cut: a name that starts with neither a blank nor `=`, the
# value everything after the first `=`, both without surrounding blanks
_ASSIGNMENT = re.compile(r"\s*([^=\s][^=]*?)\s*=\s*(.*?)\s*$")


def parse_parameters(text: str) -> dict[str, str]:
    """`{name: value}` of one SIMsalabim parameter file's text (lines without `=` are skipped)."""
    found = (_ASSIGNMENT.match(line.split("*", 1)[0]) for line in text.splitlines())
    return {m.group(1): m.group(2) for m in found if m}


@dataclass(frozen=True)
class Layer:
    """One layer's parameters as strings (SI units, energies in eV)."""

    raw: dict[str, str]

    def f(self, name: str) -> float:
        return float(self.raw[name])

    def i(self, name: str) -> int:
        return int(float(self.raw[name]))


@dataclass(frozen=True)
class Setup:
    """A simulation setup and its layers, left electrode first. A file the setup names (a
    generation profile, experimental data, a tVGFile) is taken from `files` where it is there,
    else read from `directory`."""

    raw: dict[str, str]
    layers: tuple[Layer, ...]
    directory: Path | None = None
    files: Mapping[str, str] | None = field(default=None)

    def f(self, name: str, default: float | None = None) -> float:
        """Parameter `name` as a number; `default` where the setup does not give it (one that
        only SimSS or only ZimT reads), else a KeyError."""
        if name in self.raw or default is None:
            return float(self.raw[name])
        return float(default)

    def i(self, name: str, default: int | None = None) -> int:
        return int(self.f(name, default))

    def text(self, name: str) -> str:
        """The text of the file that parameter `name` names."""
        return self.read(self.raw[name], name)

    def read(self, file: str, name: str | None = None) -> str:
        """The text of `file`; `name`, the parameter naming it, for the error."""
        if self.files is not None and file in self.files:
            return self.files[file]
        if self.directory is not None:
            return (self.directory / file).read_text()
        raise FileNotFoundError(f"{name} = {file}: not among the setup's files" if name
                                else f"{file}: not among the setup's files")


def _layers(raw: Mapping[str, str], fetch: Callable[[str], str]) -> tuple[Layer, ...]:
    """The layer files `l1`, `l2`, ... the setup names, up to the first number it does not."""
    numbers = itertools.takewhile(lambda k: f"l{k}" in raw, itertools.count(1))
    return tuple(Layer(parse_parameters(fetch(raw[f"l{k}"]))) for k in numbers)


def read_setup(path: str | os.PathLike) -> Setup:
    """A setup file and the layer files it names, found beside it."""
    path = Path(path)
    raw = parse_parameters(path.read_text())
    return Setup(raw=raw, layers=_layers(raw, lambda name: (path.parent / name).read_text()),
                 directory=path.parent)


def setup_from_texts(files: Mapping[str, str], setup: str = "simulation_setup.txt") -> Setup:
    """`read_setup` from file names mapped to their texts (the setup's own under `setup`)."""
    raw = parse_parameters(files[setup])
    return Setup(raw=raw, layers=_layers(raw, files.__getitem__), files=dict(files))


# ---------------------------------------------------------------------------------- voltages

def _measured(setup: Setup) -> np.ndarray:
    """`useExpData`: the `Vext` column of the `expJV` file, in its order."""
    table = np.genfromtxt(io.StringIO(setup.text("expJV")), names=True)
    if "Vext" not in (table.dtype.names or ()):
        raise ValueError(f"expJV = {setup.raw['expJV']}: no column Vext")
    volts = np.atleast_1d(table["Vext"]).astype(float)
    if len(volts) < 4:  # SimSS's smallest experimental curve
        raise ValueError("Not enough experimental data points (SimSS needs 4).")
    return volts


def _uniform(setup: Setup, vmin: float, vmax: float) -> np.ndarray:
    """`Vdist = 1`: from Vmin in steps of Vstep, as many as fit up to Vmax (SimSS's count,
    which takes a step within 1e-10 of fitting as fitting)."""
    step = setup.f("Vstep")
    if step <= 0:
        raise ValueError("Vstep should be positive.")
    return vmin + step * np.arange(int((vmax - vmin) / step + 1e-10) + 1)


def _accumulating(setup: Setup, vmin: float, vmax: float) -> np.ndarray:
    """`Vdist = 2`: NJV voltages from Vmin to Vmax whose distances to Vacc shrink (or grow) by
    one factor from each voltage to the next — denser toward Vacc."""
    vacc, count = setup.f("Vacc"), setup.i("NJV")
    if vmin <= vacc <= vmax:
        raise ValueError("Invalid Vacc selected, must be outside [Vmin, Vmax].")
    if abs(vmin - vmax) < 1e-10:
        raise ValueError("Do not use Vdist=2 when Vmin = Vmax.")
    if count < 2:
        raise ValueError(f"NJV = {count}: Vdist = 2 needs at least 2 voltages")
    first, final = vacc - vmin, vacc - vmax  # the distances to Vacc at both ends
    return vacc - first * (final / first) ** (np.arange(count) / (count - 1))


_GRIDS: dict[int, Callable[[Setup, float, float], np.ndarray]] = {1: _uniform, 2: _accumulating}


def simss_voltages(setup: Setup) -> np.ndarray:
    """The internal voltages SimSS simulates, in its order: `Vdist` 1 (uniform) or 2
    (accumulating toward `Vacc`) from `Vmin` to `Vmax`, reversed for `Vscan = -1`; with
    `useExpData` the `Vext` column of `expJV` instead. The pre-bias is not among them. SimSS's
    checks raise `ValueError`."""
    if int(float(setup.raw.get("useExpData", "0"))):
        return _measured(setup)
    dist, scan = setup.i("Vdist"), setup.i("Vscan")
    vmin, vmax = setup.f("Vmin"), setup.f("Vmax")
    if dist not in _GRIDS:
        raise ValueError(f"Vdist = {dist}: SimSS has 1 (uniform) and 2 (logarithmic)")
    if scan not in (-1, 1):
        raise ValueError("Vscan must be either -1 or 1.")
    if vmin > vmax:
        raise ValueError("Vmin should not be greater than Vmax.")
    volts = _GRIDS[dist](setup, vmin, vmax)
    return np.ascontiguousarray(volts[::-1]) if scan == -1 else volts


# ---------------------------------------------------------------------------------- tVGFile

#: ln of the largest real SIMsalabim's Pascal code handles (extended precision): the voltage's
#: bound in `read_tvg`, |V/V_T| < 1.95 of it.
LN_MAX_EXTENDED = 11356.523406294143


@dataclass(frozen=True)
class TVG:
    """ZimT's time steps (`tVGFile`): at each time `t` (s) the voltage `Vext` (V; NaN where
    `oc`, the open circuit), `G_frac` and `track` (0–3, ZimT's automatic stop); `dti` 1/Δt from
    the step before, 0 at `t = 0` (a steady state). With them the setup's `failureMode` (0 stop
    at a failed step, 1 keep it, 2 skip it), `convVar` and the tolerances that compare two states
    (`tolPois` V, `tolDens`, `tolCurr` A/m²)."""

    t: np.ndarray
    Vext: np.ndarray
    oc: np.ndarray
    G_frac: np.ndarray
    track: np.ndarray
    dti: np.ndarray
    failure_mode: int = 1
    conv_var: int = 1
    tol_pois: float = 1e-6
    tol_dens: float = 1e-6
    tol_curr: float = 1e-3

    @classmethod
    def steps(cls, t, Vext, G_frac=1.0, track=0, failure_mode: int = 1) -> "TVG":
        """Time steps from arrays (the first at `t = 0`), as `read_tvg` would read them."""
        times = np.asarray(t, dtype=float)
        n = len(times)
        if n == 0 or times[0] != 0:
            raise ValueError("tVGFile did not specify steady-state (t=0)")
        dti = np.array([_inverse_step(b, a) for a, b in zip(np.r_[0.0, times[:-1]], times)])
        full = [np.broadcast_to(np.asarray(a), (n,)).copy() for a in (Vext, G_frac, track)]
        return cls(t=times, Vext=full[0].astype(float), oc=np.zeros(n, bool),
                   G_frac=full[1].astype(float), track=full[2].astype(int), dti=dti,
                   failure_mode=int(failure_mode))


def _inverse_step(t: float, previous: float) -> float:
    """1/Δt of a step at `t` after one at `previous`, 0 for a return to t = 0; ZimT refuses a
    time that goes back to anything but 0."""
    if t > previous:
        return 1.0 / (t - previous)
    if t == 0:
        return 0.0
    raise ValueError("Time steps must either be positive, or you should go back to t=0 "
                     f"(steady-state); at t = {t}")


def _tvg_lines(text: str, name: str) -> Iterator[str]:
    """The step lines of a tVGFile: after its header `t Vext G_frac Track` (blanks and case
    ignored), up to its end or its first empty line."""
    lines = iter(text.splitlines())
    if not any("".join(line.lower().split()).startswith("tvextg_fractrack") for line in lines):
        raise ValueError(f"Could not find correct header 't Vext G_frac Track' in {name}.")
    return itertools.takewhile(lambda line: line.split() != [], lines)


def read_tvg(setup: Setup) -> TVG:
    """ZimT 5.36's `tVGFile`: one step per line (`t`, `Vext` or `oc`, `G_frac`, `Track`; columns
    past the fourth ignored). ZimT's checks raise `ValueError`, each at the first line that
    breaks it, in ZimT's order: the line's numbers, its time (forward, or back to 0), its voltage
    within SIMsalabim's range, a `Track` of 2 or 3 only after a 1 — one on the first line does
    not count, ZimT forgets it — and, once read, a first step at `t = 0`, `failureMode` and
    `convVar` among ZimT's."""
    from jaxdd_b200.constants import K_B, Q

    name = setup.raw["tVGFile"]
    volts_per_vt = Q / (K_B * setup.f("T"))
    columns: dict[str, list] = {k: [] for k in ("t", "Vext", "oc", "G_frac", "track", "dti")}
    reference_set = False
    for line in _tvg_lines(setup.text("tVGFile"), name):
        t_text, v_text, g_text, track = (line.split() + ["", "", "", ""])[:4]
        try:
            t, g = float(t_text), float(g_text)
            open_circuit = v_text.lower() == "oc"
            v = float("nan") if open_circuit else float(v_text)
            if track not in {"0", "1", "2", "3"}:
                raise ValueError
        except ValueError:
            raise ValueError(f"Error while reading from file {name}; offending line: {line!r}") \
                from None
        dti = _inverse_step(t, columns["t"][-1] if columns["t"] else 0.0)
        if not open_circuit and abs(v * volts_per_vt) > 1.95 * LN_MAX_EXTENDED:
            raise ValueError(f"V is too {'small' if v < 0 else 'large'}; at t = {t}")
        reference_set = reference_set or (track == "1" and bool(columns["t"]))
        if track in {"2", "3"} and not reference_set:
            raise ValueError("Error in tVGFile: before setting Track=2 or 3, you need to have at "
                             "least one Track=1")
        for key, value in zip(columns, (t, v, open_circuit, g, int(track), dti)):
            columns[key].append(value)
    if not columns["t"] or columns["t"][0] != 0:
        raise ValueError("tVGFile did not specify steady-state (t=0)")
    failure_mode = int(setup.raw.get("failureMode", 1))
    conv_var = int(setup.raw.get("convVar", 1))
    if failure_mode not in {0, 1, 2}:
        raise ValueError("Invalid failureMode selected.")
    if conv_var not in {1, 2, 3, 4}:
        raise ValueError("Invalid convVar selected.")
    kinds = {"t": float, "Vext": float, "oc": bool, "G_frac": float, "track": int, "dti": float}
    return TVG(**{k: np.array(v, dtype=kinds[k]) for k, v in columns.items()},
               failure_mode=failure_mode, conv_var=conv_var,
               tol_pois=float(setup.raw.get("tolPois", 1e-6)),
               tol_dens=float(setup.raw.get("tolDens", 1e-6)),
               tol_curr=float(setup.raw.get("tolCurr", 1e-3)))


# ---------------------------------------------------------------------------------- ions

def ion_regions(setup: Setup, species: str) -> list[tuple[int, int, bool]]:
    """SIMsalabim's ionic regions of one species (`Init_Ionic_Region`): `(first, last, mobile)`
    layer indices. The layers that can hold ions — those the ions may enter, and a layer of
    immobile ions — form runs; within a run a region closes at a layer whose ions do not move or
    before a layer they may not enter, counts if the ions it took in are not zero, and is mobile
    when its last layer's mobility is not zero. As SimSS 5.36 has it, a region that closes does
    not move the start: the next region of the same run starts where the run does. SimSS's
    check: a layer with mobile ions must let them enter."""
    layers = setup.layers
    mu = [ly.f(f"mu_{species}") for ly in layers]
    conc = [ly.f(f"N_{species}") for ly in layers]
    enter = [bool(ly.i("ionsMayEnter")) for ly in layers]
    for j in range(len(layers)):
        if mu[j] * conc[j] > 0 and not enter[j]:
            raise ValueError(f"layer {j + 1}: If a layer contains mobile ions, then ionsMayEnter "
                             "(of that layer) must be 1.")
    holds = [enter[j] or (mu[j] == 0 and conc[j] > 0) for j in range(len(layers))]
    found: list[tuple[int, int, bool]] = []
    j = 0
    while j < len(layers):
        if not holds[j]:
            j += 1
            continue
        run_start, taken = j, 0.0
        while j < len(layers) and holds[j]:
            taken += layers[j].f("L") * conc[j]
            if j + 1 == len(layers) or not enter[j + 1] or mu[j] == 0:
                if taken != 0:
                    found.append((run_start, j, mu[j] > 0))
                taken = 0.0
            j += 1
    return found


def ion_region_problems(setup: Setup) -> list[str]:
    """SimSS 5.36's two ways of solving a region of several layers against what the input says
    (a layer the ions may not enter taken in; a last layer of mobility 0 holding them all),
    which jaxdd refuses."""
    found = []
    for species in ("anion", "cation"):
        for first, last, mobile in ion_regions(setup, species):
            span = range(first, last + 1)
            if first == last:
                continue
            where = f"{species}s: SimSS's region of layers {first + 1}–{last + 1}"
            closed = [k + 1 for k in span if not setup.layers[k].i("ionsMayEnter")]
            if closed:
                found.append(f"{where} takes in layer {closed[0]}, which they may not enter")
            moving = any(setup.layers[k].f(f"mu_{species}") * setup.layers[k].f(f"N_{species}")
                         > 0 for k in span)
            if not mobile and moving:
                found.append(f"{where} has mobility 0 in its last layer, so it holds them all")
    return found


def check_supported(setup: Setup) -> None:
    """Raise `NotImplementedError` naming what SimSS itself refuses and the ionic regions jaxdd
    refuses (`ion_region_problems`). What this build leaves out beyond that is refused by
    `device.build_device`, by name."""
    raw = setup.raw
    found = []
    if float(raw.get("currDiffInt", 2)) not in (1.0, 2.0):
        found.append(f"currDiffInt = {raw['currDiffInt']} (SimSS has 1 and 2)")
    if float(raw.get("R_series", 0)) < 0 or float(raw.get("R_shunt", -1)) == 0:
        found.append("R_series < 0 or R_shunt = 0 (SimSS refuses both)")
    found.extend(ion_region_problems(setup))
    if found:
        raise NotImplementedError("outside what jaxdd solves:\n  " + "\n  ".join(found))
