"""SIMsalabim input files: `simulation_setup.txt` and the layer files it names.

Same file format and the same public functions as jaxdd's reader (jaxdd src/jaxdd/simss_input.py):
each line `name = value * comment`, `*` starting a comment, names in any order. Values stay
strings until a consumer converts them, so that an unsupported parameter can be refused by
name (`check_supported`).
"""

from __future__ import annotations

import io
import os
from collections.abc import Mapping
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

__all__ = [
    "Layer",
    "Setup",
    "check_supported",
    "ion_regions",
    "parse_parameters",
    "read_setup",
    "setup_from_texts",
    "simss_voltages",
]


def parse_parameters(text: str) -> dict[str, str]:
    """`{name: value}` of one parameter file (jaxdd simss_input.py:40-50)."""
    out: dict[str, str] = {}
    for raw_line in text.splitlines():
        content = raw_line.partition("*")[0]
        name, eq, value = content.partition("=")
        if not eq:
            continue
        name = name.strip()
        if name:
            out[name] = value.strip()
    return out


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
    """A simulation setup with its layers (left electrode first). Files it names (the generation
    profile) come from `files` if given there, else from `directory` (jaxdd simss_input.py:68-107)."""

    raw: dict[str, str]
    layers: tuple[Layer, ...]
    directory: Path | None = None
    files: Mapping[str, str] | None = field(default=None)

    def f(self, name: str, default: float | None = None) -> float:
        if default is not None and name not in self.raw:
            return float(default)
        return float(self.raw[name])

    def i(self, name: str, default: int | None = None) -> int:
        return int(self.f(name, default))

    def text(self, name: str) -> str:
        return self.read(self.raw[name], name)

    def read(self, file: str, name: str | None = None) -> str:
        if self.files is not None and file in self.files:
            return self.files[file]
        if self.directory is None:
            label = f"{name} = {file}" if name else file
            raise FileNotFoundError(f"{label}: not among the setup's files")
        return (self.directory / file).read_text()


def _read_layers(raw: Mapping[str, str], fetch) -> tuple[Layer, ...]:
    layers = []
    k = 1
    while f"l{k}" in raw:
        layers.append(Layer(parse_parameters(fetch(raw[f"l{k}"]))))
        k += 1
    return tuple(layers)


def read_setup(path: str | os.PathLike) -> Setup:
    """A setup file and the layer files `l1`, `l2`, ... beside it (jaxdd simss_input.py:277-282)."""
    path = Path(path)
    raw = parse_parameters(path.read_text())
    return Setup(raw=raw, layers=_read_layers(raw, lambda f: (path.parent / f).read_text()),
                 directory=path.parent)


def setup_from_texts(files: Mapping[str, str], setup: str = "simulation_setup.txt") -> Setup:
    """`read_setup` from a mapping of file names to texts (jaxdd simss_input.py:285-289)."""
    raw = parse_parameters(files[setup])
    return Setup(raw=raw, layers=_read_layers(raw, lambda f: files[f]), files=dict(files))


def simss_voltages(setup: Setup) -> np.ndarray:
    """The internal voltages SimSS runs (`Vdist` 1 uniform by `Vstep`, 2 accumulating towards
    `Vacc`), reversed for `Vscan = -1`, or the `Vext` column of `expJV` with `useExpData`
    (jaxdd simss_input.py:108-145). SimSS's own checks raise `ValueError`."""
    if int(float(setup.raw.get("useExpData", "0"))):
        table = np.genfromtxt(io.StringIO(setup.text("expJV")), names=True)
        if "Vext" not in (table.dtype.names or ()):
            raise ValueError(f"expJV = {setup.raw['expJV']}: no column Vext")
        v = np.atleast_1d(table["Vext"]).astype(float)
        if v.size < 4:
            raise ValueError("Not enough experimental data points (SimSS needs 4).")
        return v
    vdist, vscan = setup.i("Vdist"), setup.i("Vscan")
    vmin, vmax = setup.f("Vmin"), setup.f("Vmax")
    if vdist not in (1, 2):
        raise ValueError(f"Vdist = {vdist}: SimSS has 1 (uniform) and 2 (logarithmic)")
    if abs(vscan) != 1:
        raise ValueError("Vscan must be either -1 or 1.")
    if vmin > vmax:
        raise ValueError("Vmin should not be greater than Vmax.")
    if vdist == 1:
        step = setup.f("Vstep")
        if step <= 0:
            raise ValueError("Vstep should be positive.")
        count = int(np.trunc((vmax - vmin) / step + 1e-10)) + 1
        v = vmin + step * np.arange(count)
    else:
        acc, count = setup.f("Vacc"), setup.i("NJV")
        if vmin <= acc <= vmax:
            raise ValueError("Invalid Vacc selected, must be outside [Vmin, Vmax].")
        if abs(vmin - vmax) < 1e-10:
            raise ValueError("Do not use Vdist=2 when Vmin = Vmax.")
        if count < 2:
            raise ValueError(f"NJV = {count}: Vdist = 2 needs at least 2 voltages")
        d = acc - vmax
        v = acc - d * np.exp((1 - np.arange(count) / (count - 1)) * np.log((acc - vmin) / d))
    return v[::-1].copy() if vscan == -1 else v


def ion_regions(setup: Setup, species: str) -> list[tuple[int, int, bool]]:
    """SIMsalabim's ionic regions of one species (`Init_Ionic_Region`): `(first, last, mobile)`
    layer indices. A region is a run of layers the ions may enter (or one layer of immobile
    ions) that holds ions; it closes at a layer whose ions do not move or before a layer they may
    not enter, and is mobile when its last layer's mobility is not zero. As SimSS 5.36, a region
    that follows directly starts where the one before started (jaxdd simss_input.py:226-253)."""
    found: list[tuple[int, int, bool]] = []
    start: int | None = None
    held = 0.0
    layers = setup.layers
    for j, layer in enumerate(layers):
        mu, conc = layer.f(f"mu_{species}"), layer.f(f"N_{species}")
        enter = layer.i("ionsMayEnter")
        if mu * conc > 0 and not enter:
            raise ValueError(f"layer {j + 1}: If a layer contains mobile ions, then ionsMayEnter "
                             "(of that layer) must be 1.")
        if not (enter or (mu == 0 and conc > 0)):
            start, held = None, 0.0
            continue
        held += layer.f("L") * conc
        if start is None:
            start = j
        closes = j == len(layers) - 1 or not layers[j + 1].i("ionsMayEnter") or mu == 0
        if closes:
            if held != 0:
                found.append((start, j, mu > 0))
            held = 0.0
    return found


def ion_region_problems(setup: Setup) -> list[str]:
    """The two multi-layer ionic regions SimSS 5.36 solves against what the input says, which
    jaxdd refuses (jaxdd simss_input.py:292-308)."""
    out = []
    for species in ("anion", "cation"):
        for first, last, mobile in ion_regions(setup, species):
            if first == last:
                continue
            span = setup.layers[first:last + 1]
            where = f"{species}s: SimSS's region of layers {first + 1}–{last + 1}"
            closed = [first + 1 + k for k, ly in enumerate(span) if not ly.i("ionsMayEnter")]
            if closed:
                out.append(f"{where} takes in layer {closed[0]}, which they may not enter")
            if not mobile and any(ly.f(f"mu_{species}") * ly.f(f"N_{species}") > 0 for ly in span):
                out.append(f"{where} has mobility 0 in its last layer, so it holds them all")
    return out


def check_supported(setup: Setup) -> None:
    """Raise `NotImplementedError` naming what SimSS itself refuses (jaxdd
    simss_input.py:311-333). What this build leaves out beyond that is refused by
    `device.build_device`, by name."""
    problems = []
    if float(setup.raw.get("currDiffInt", 2)) not in (1.0, 2.0):
        problems.append(f"currDiffInt = {setup.raw['currDiffInt']} (SimSS has 1 and 2)")
    if float(setup.raw.get("R_series", 0)) < 0 or float(setup.raw.get("R_shunt", -1)) == 0:
        problems.append("R_series < 0 or R_shunt = 0 (SimSS refuses both)")
    problems += ion_region_problems(setup)
    if problems:
        raise NotImplementedError("outside what jaxdd solves:\n  " + "\n  ".join(problems))
