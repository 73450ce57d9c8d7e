"""Run MD from a FeNNol ``.fnl`` input file on the CUDA path.

    python -m fennol_b200.md_driver input.fnl

Reads the keys of FeNNol's MD input (``src/fennol/md/dynamic.py``,
``md/initial.py``, parsed as ``utils/input_parser.py`` does: ``key value``
or ``key = value`` lines, ``name{ ... }`` sections, ``#``/``!`` comments,
units in brackets ``dt[fs]`` or braces ``gamma{THz}``) and drives
:class:`fennol_b200.md.MDEngine`:

* ``model_file`` (a ``.fnx`` / ``.pkl`` written by ``FENNIX.save``), or
  ``random_model_seed`` for a seeded random ANI-2x-style network;
* ``xyz_input{ file, indexed, has_comment_line }``, ``cell`` (9 numbers,
  rows are lattice vectors), ``minimum_image``;
* ``nsteps``, ``dt``, ``nblist_skin``, ``thermostat`` (``NVE`` or ``LGV``),
  ``temperature``, ``gamma``;
* ``traj_format`` (``xyz``, ``arc``, ``extxyz``), ``tdump``, ``nprint``;
* ``matmul_prec`` (``highest`` → FP32 MLP, otherwise split-BF16 tensor
  cores) or ``precision`` (``fp32``, ``bf16x2``, ``bf16x3``).

Unsupported thermostats and features (QTB, PIMD beads, barostats) raise.
"""

from __future__ import annotations

import math
import re
import sys
import time
from pathlib import Path
from typing import Any, Dict

import numpy as np

# multipliers to the MD units used here: fs for dt, ps for times, 1/ps for
# frequencies, K, Angstrom
_UNITS = {
    "fs": ("time", 1e-3), "ps": ("time", 1.0), "ns": ("time", 1e3),
    "thz": ("freq", 1.0), "ps-1": ("freq", 1.0), "ps^-1": ("freq", 1.0), "fs-1": ("freq", 1e3),
    "k": ("temp", 1.0), "kelvin": ("temp", 1.0),
    "a": ("length", 1.0), "ang": ("length", 1.0), "angstrom": ("length", 1.0),
    "bohr": ("length", 0.52917721),
}
_TRUE = {"true", "yes", ".true."}
_FALSE = {"false", "no", ".false."}


def _value(tokens):
    vals = []
    for t in tokens:
        low = t.lower()
        if low in _TRUE:
            vals.append(True)
        elif low in _FALSE:
            vals.append(False)
        else:
            try:
                vals.append(int(t))
            except ValueError:
                try:
                    vals.append(float(t))
                except ValueError:
                    vals.append(t)
    if not vals:
        return True  # a bare key is a flag
    return vals[0] if len(vals) == 1 else vals


def parse_fnl(text: str) -> Dict[str, Any]:
    """Parameters of a ``.fnl`` text as a nested dict with lower-case keys.
    A key with a unit (``dt[fs]``) is stored as ``(value, unit)``."""
    root: Dict[str, Any] = {}
    stack = [root]
    for raw in text.splitlines():
        line = raw
        for ch in "#!":
            if ch in line:
                line = line[:line.index(ch)]
        line = line.strip()
        if not line:
            continue
        if line == "}":
            if len(stack) == 1:
                raise ValueError("unbalanced '}' in input")
            stack.pop()
            continue
        if line.endswith("{"):
            name = line[:-1].strip().lower()
            sec: Dict[str, Any] = {}
            stack[-1][name] = sec
            stack.append(sec)
            continue
        parts = [p for p in re.split(r"[\s=,]+", line) if p]
        key, tokens = parts[0], parts[1:]
        m = re.fullmatch(r"([^\[\{]+)[\[\{]([^\]\}]+)[\]\}]", key)
        val = _value(tokens)
        if m:
            stack[-1][m.group(1).lower()] = (val, m.group(2).strip())
        else:
            stack[-1][key.lower()] = val
    if len(stack) != 1:
        raise ValueError("unclosed section in input")
    return root


def get(params: Dict[str, Any], key: str, default=None, kind: str = None):
    """A parameter with its unit converted (``kind``: time→ps, freq→1/ps,
    temp→K, length→A)."""
    node = params
    for part in key.lower().split("/"):
        if not isinstance(node, dict) or part not in node:
            return default
        node = node[part]
    if isinstance(node, tuple):
        val, unit = node
        u = _UNITS.get(unit.lower())
        if u is None or (kind is not None and u[0] != kind):
            raise ValueError(f"unit {unit!r} of {key} not understood")
        return val * u[1]
    return node


def read_xyz_input(path: str, indexed: bool, has_comment_line: bool):
    """Species (atomic numbers) and coordinates of the first frame of an xyz
    or Tinker-style file (``indexed``: a leading atom index column)."""
    from .params import PERIODIC_TABLE_REV_IDX
    lines = Path(path).read_text().splitlines()
    n = int(lines[0].split()[0])
    body = lines[2:2 + n] if has_comment_line else lines[1:1 + n]
    sym, xyz = [], []
    for ln in body:
        t = ln.split()
        if indexed:
            t = t[1:]
        sym.append(t[0])
        xyz.append([float(v) for v in t[1:4]])
    z = np.array([PERIODIC_TABLE_REV_IDX[s.capitalize() if len(s) > 1 else s.upper()] for s in sym])
    return z, np.array(xyz)


def run(params: Dict[str, Any], workdir: Path, out=sys.stdout):
    import torch

    from .fennix import FENNIX
    from .md import MDEngine
    from .params import AEVConfig, MLPConfig, init_weights
    from .potential import ANIPotential
    from .trajectory import FrameStream

    for key in ("nbeads", "qtb", "barostat"):
        if get(params, key) is not None:
            raise NotImplementedError(f"'{key}' is outside the CUDA MD path")
    thermostat = str(get(params, "thermostat", "LGV")).upper()
    if thermostat not in ("LGV", "LANGEVIN", "NVE"):
        raise NotImplementedError(f"thermostat {thermostat} is outside the CUDA MD path")
    prec = get(params, "precision")
    if prec is None:
        prec = "fp32" if str(get(params, "matmul_prec", "highest")).lower() == "highest" else "bf16x3"
    device = str(get(params, "device", "cuda:0"))
    if not device.startswith("cuda"):
        raise NotImplementedError("the CUDA MD path runs on a CUDA device")
    model_file = get(params, "model_file")
    if model_file is not None:
        model = FENNIX.load(workdir / str(model_file), precision=prec, device=device)
        pot = ANIPotential(model.aev_config, model.mlp_config, weights=model.weights(),
                           precision=prec, device=device)
    else:
        seed = int(get(params, "random_model_seed", 0))
        scale = float(get(params, "random_model_output_scale", 0.02))
        cfg, mcfg = AEVConfig(), MLPConfig()
        pot = ANIPotential(cfg, mcfg, weights=init_weights(cfg, mcfg, seed=seed, output_scale=scale),
                           precision=prec, device=device)
    xin = get(params, "xyz_input", {})
    species, coords = read_xyz_input(str(workdir / str(xin.get("file"))), bool(xin.get("indexed", False)),
                                     bool(xin.get("has_comment_line", True)))
    cell = get(params, "cell")
    if cell is not None:
        cell = np.asarray(cell, dtype=np.float64).reshape(3, 3)
        mi = get(params, "minimum_image", None)
        if mi is not None:
            pot.minimum_image = bool(mi)
    dt_fs = get(params, "dt", 0.5, "time") * 1000.0
    nsteps = int(get(params, "nsteps", 1000))
    skin = float(get(params, "nblist_skin", 1.0, "length"))
    temperature = float(get(params, "temperature", 300.0, "temp"))
    gamma = float(get(params, "gamma", 1.0, "freq"))
    eng = MDEngine(pot, coords, species, cell, dt_fs=dt_fs, thermostat=thermostat,
                   temperature=temperature, gamma_ps=gamma, skin=skin, seed=int(get(params, "seed", 0)))
    nprint = max(1, int(get(params, "nprint", 100)))
    fmt = str(get(params, "traj_format", "arc")).lower()
    tdump = get(params, "tdump", None, "time")
    dump_every = max(1, int(round(tdump / eng.dt))) if tdump else 0
    stem = Path(str(xin.get("file"))).stem
    frames = FrameStream(str(workdir / f"{stem}.traj.{fmt}"), species, fmt, cell) if dump_every else None
    print(f"# {len(species)} atoms, {nsteps} steps of {dt_fs} fs, {thermostat}, precision {prec}", file=out)
    print(f"# {'step':>8} {'time[ps]':>10} {'Epot[kcal/mol]':>16} {'Ekin[kcal/mol]':>16} "
          f"{'Etot[kcal/mol]':>16} {'T[K]':>8} {'ns/day':>8}", file=out)
    done, t0 = 0, time.perf_counter()
    chunk = math.gcd(nprint, dump_every) if dump_every else nprint
    while done < nsteps:
        k = min(chunk, nsteps - done)
        eng.run(k, sync=False)
        done += k
        if frames is not None and done % dump_every == 0:
            frames.push(eng.x, properties={"time_ps": f"{eng.simulation_time_ps():.6f}"})
        if done % nprint == 0 or done == nsteps:
            ep, ek = eng.potential_energy(), eng.kinetic_energy()
            el = time.perf_counter() - t0
            nsday = eng.simulation_time_ps() * 1e-3 / max(el, 1e-9) * 86400.0
            print(f"  {done:>8d} {eng.simulation_time_ps():>10.4f} {ep:>16.4f} {ek:>16.4f} {ep + ek:>16.4f} "
                  f"{eng.temperature():>8.2f} {nsday:>8.2f}", file=out)
    if frames is not None:
        frames.close()
    torch.cuda.synchronize(pot.device)
    if get(params, "write_restart", True):
        eng.save_restart(str(workdir / f"{stem}.dyn.restart"))
    return eng


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if not argv:
        print(__doc__)
        return 2
    path = Path(argv[0])
    run(parse_fnl(path.read_text()), path.parent)
    return 0


if __name__ == "__main__":
    sys.exit(main())
