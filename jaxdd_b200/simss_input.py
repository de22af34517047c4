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
    "TVG",
    "check_supported",
    "ion_regions",
    "parse_parameters",
    "read_setup",
    "read_tvg",
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


#: ln of the largest real SIMsalabim's Pascal code handles (extended precision): the voltage's
#: bound in `read_tvg`, |V/V_T| < 1.95 of it.
LN_MAX_EXTENDED = 11356.523406294143


@dataclass(frozen=True)
class TVG:
    """ZimT's time steps (`tVGFile`, jaxdd simss_input.py:155-175): at each time `t` (s) the
    voltage `Vext` (V; NaN where `oc`, the open circuit), `G_frac` and `track` (0–3, ZimT's
    automatic stop); `dti` 1/Δt from the step before, 0 at `t = 0` (a steady state). With
    them the setup's `failureMode` (0 stop at a failed step, 1 keep it, 2 skip it), `convVar`
    and the tolerances that compare two states (`tolPois` V, `tolDens`, `tolCurr` A/m²)."""

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
        t = np.asarray(t, dtype=float)
        n = t.shape[0]
        Vext, G_frac, track = (np.broadcast_to(np.asarray(a), (n,)).copy()
                               for a in (Vext, G_frac, track))
        if n == 0 or t[0] != 0:
            raise ValueError("tVGFile did not specify steady-state (t=0)")
        dti, previous = np.zeros(n), 0.0
        for k, tk in enumerate(t):
            if tk > previous:
                dti[k] = 1.0 / (tk - previous)
            elif tk != 0:
                raise ValueError("Time steps must either be positive, or you should go back to "
                                 f"t=0 (steady-state); at t = {tk}")
            previous = tk
        return cls(t=t, Vext=Vext.astype(float), oc=np.zeros(n, bool),
                   G_frac=G_frac.astype(float), track=track.astype(int), dti=dti,
                   failure_mode=int(failure_mode))


def read_tvg(setup: Setup) -> TVG:
    """ZimT 5.36's `tVGFile` (jaxdd simss_input.py:178-237): lines up to the header
    `t Vext G_frac Track` skipped, then one step per line up to the end or an empty line,
    columns past the fourth ignored. ZimT's checks raise `ValueError`: the header, a first step
    at `t = 0`, times that go forward or back to 0, a voltage within range, `Track` 0–3 with a
    1 (not on the first line, which ZimT forgets) before any 2 or 3."""
    name = setup.raw["tVGFile"]
    lines = iter(setup.text("tVGFile").splitlines())
    for line in lines:
        if "".join(line.lower().split()).startswith("tvextg_fractrack"):
            break
    else:
        raise ValueError(f"Could not find correct header 't Vext G_frac Track' in {name}.")
    from jaxdd_b200.constants import K_B, Q

    vti = Q / (K_B * setup.f("T"))
    rows: list[tuple] = []
    previous, seen_one = 0.0, False
    for line in lines:
        words = line.split()
        if not words:
            break
        t_s, v_s, g_s, track_s = (words + [""] * 4)[:4]
        try:
            t, g = float(t_s), float(g_s)
            oc = v_s.lower() == "oc"
            v = np.nan if oc else float(v_s)
            if track_s not in ("0", "1", "2", "3"):
                raise ValueError
        except ValueError:
            raise ValueError(f"Error while reading from file {name}; offending line: {line!r}") \
                from None
        if t > previous:
            dti = 1.0 / (t - previous)
        elif t == 0:
            dti = 0.0
        else:
            raise ValueError("Time steps must either be positive, or you should go back to t=0 "
                             f"(steady-state); at t = {t}")
        if not oc and abs(v * vti) > 1.95 * LN_MAX_EXTENDED:
            raise ValueError(f"V is too {'small' if v < 0 else 'large'}; at t = {t}")
        if rows and track_s == "1":
            seen_one = True
        if track_s in ("2", "3") and not seen_one:
            raise ValueError("Error in tVGFile: before setting Track=2 or 3, you need to have at "
                             "least one Track=1")
        rows.append((t, v, oc, g, int(track_s), dti))
        previous = t
    if not rows or rows[0][0] != 0:
        raise ValueError("tVGFile did not specify steady-state (t=0)")
    t, v, oc, g, track, dti = (np.array(c) for c in zip(*rows))
    failure_mode, conv_var = int(setup.raw.get("failureMode", 1)), int(setup.raw.get("convVar", 1))
    if failure_mode not in (0, 1, 2):
        raise ValueError("Invalid failureMode selected.")
    if conv_var not in (1, 2, 3, 4):
        raise ValueError("Invalid convVar selected.")
    return TVG(t=t.astype(float), Vext=v.astype(float), oc=oc.astype(bool),
               G_frac=g.astype(float), track=track.astype(int), dti=dti.astype(float),
               failure_mode=failure_mode, conv_var=conv_var,
               tol_pois=float(setup.raw.get("tolPois", 1e-6)),
               tol_dens=float(setup.raw.get("tolDens", 1e-6)),
               tol_curr=float(setup.raw.get("tolCurr", 1e-3)))


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
