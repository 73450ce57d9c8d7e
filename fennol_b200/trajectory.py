"""Trajectory files and restarts from device-resident MD state.

Frames are written in the formats FeNNol's MD driver writes
(``src/fennol/utils/io.py:121-185``, called from ``md/dynamic.py:530-592``):

* ``xyz``: atom count, a comment line with the cell as lengths and angles
  (empty without a cell), then ``symbol x y z``;
* ``arc`` (Tinker): atom count, the cell line, then ``index symbol x y z``;
* ``extxyz``: atom count, ``Lattice="..." Properties=species:S:1:pos:R:3``
  (``:forces:R:3`` with forces) plus ``key=value`` properties, then the rows.

:class:`FrameStream` copies positions out of the device with asynchronous
copies into pinned host buffers on a side stream, so the MD stream keeps
running while the previous frame is formatted and written.

Restart files are pickles of the keys ``save_dynamics_restart`` writes
(``md/utils.py:36-55``): ``nat``, ``species``, ``coordinates``, ``vel``,
``simulation_time_ps`` and ``cells`` for periodic systems.
"""

from __future__ import annotations

import math
import pickle
from typing import Dict, Optional, Sequence

import numpy as np
import torch

from .params import PERIODIC_TABLE


def cell_lengths_angles(cell) -> np.ndarray:
    """(a, b, c, alpha, beta, gamma) of a cell whose rows are the lattice
    vectors; angles in degrees."""
    c = np.asarray(cell, dtype=np.float64).reshape(3, 3)
    a, b, cc = (float(np.linalg.norm(c[k])) for k in range(3))

    def angle(u, v):
        return math.degrees(math.acos(float(np.clip(np.dot(u, v) / (np.linalg.norm(u) * np.linalg.norm(v)),
                                                    -1.0, 1.0))))

    return np.array([a, b, cc, angle(c[1], c[2]), angle(c[0], c[2]), angle(c[0], c[1])])


def symbols_of(species) -> list:
    return [PERIODIC_TABLE[int(z)] for z in np.asarray(species)]


def _rows(fmt_row: str, symbols, values: np.ndarray) -> str:
    return "".join(fmt_row.format(s, *v) for s, v in zip(symbols, values.tolist()))


def format_frame(fmt: str, symbols: Sequence[str], coordinates: np.ndarray, cell=None,
                 forces: Optional[np.ndarray] = None, properties: Optional[Dict] = None) -> str:
    """One frame as text in ``xyz``, ``arc`` or ``extxyz`` format."""
    x = np.asarray(coordinates, dtype=np.float64).reshape(-1, 3)
    nat = x.shape[0]
    if fmt == "xyz":
        head = f"{nat}\n"
        head += (" ".join(f"{v:.3f}" for v in cell_lengths_angles(cell)) if cell is not None else "") + "\n"
        return head + _rows("{:3} {: 15.5e} {: 15.5e} {: 15.5e}\n", symbols, x)
    if fmt == "arc":
        head = f"{nat}\n"
        if cell is not None:
            head += " ".join(f"{v: 15.5f}" for v in cell_lengths_angles(cell)) + "\n"
        idx = [f"{k + 1} {s:3}" for k, s in enumerate(symbols)]
        return head + _rows("{} {: 15.3f} {: 15.3f} {: 15.3f}\n", idx, x)
    if fmt == "extxyz":
        comment = ""
        if cell is not None:
            comment += 'Lattice="' + " ".join(f"{v:.3f}" for v in np.asarray(cell).reshape(-1)) + '" '
        comment += "Properties=species:S:1:pos:R:3"
        rows = x
        fmt_row = "{:3} {: 15.5e} {: 15.5e} {: 15.5e}\n"
        if forces is not None:
            comment += ":forces:R:3"
            rows = np.concatenate([x, np.asarray(forces, np.float64).reshape(-1, 3)], axis=1)
            fmt_row = "{:3} {: 15.5e} {: 15.5e} {: 15.5e} {: 15.5e} {: 15.5e} {: 15.5e}\n"
        comment += " " + "".join(f"{k}={v} " for k, v in (properties or {}).items())
        return f"{nat}\n{comment}\n" + _rows(fmt_row, symbols, rows)
    raise ValueError(f"unknown trajectory format {fmt!r}")


def read_xyz(path: str):
    """Frames of an xyz / extxyz file as (symbols, coordinates [n, 3], comment)."""
    frames = []
    with open(path) as f:
        lines = f.read().splitlines()
    k = 0
    while k < len(lines):
        if not lines[k].strip():
            k += 1
            continue
        n = int(lines[k])
        comment = lines[k + 1]
        rows = [ln.split() for ln in lines[k + 2:k + 2 + n]]
        frames.append(([r[0] for r in rows], np.array([[float(v) for v in r[1:4]] for r in rows]), comment))
        k += 2 + n
    return frames


class FrameStream:
    """Writes frames of a device tensor without stalling the stream that
    produces it: each frame is copied into a pinned buffer on a side stream
    and written to the file when the next frame is requested (or on close)."""

    def __init__(self, path: str, species, fmt: str = "xyz", cell=None):
        self.f = open(path, "w")
        self.fmt, self.cell = fmt, cell
        self.symbols = symbols_of(species)
        self.copy_stream = None
        self.pending = None
        self.frames = 0

    def push(self, coords: torch.Tensor, properties: Optional[Dict] = None):
        """Queue the current contents of ``coords`` ([N, 3] on the device)."""
        self._drain()
        if self.copy_stream is None:
            self.copy_stream = torch.cuda.Stream(coords.device)
        host = torch.empty(tuple(coords.shape), dtype=coords.dtype, pin_memory=True)
        self.copy_stream.wait_stream(torch.cuda.current_stream(coords.device))
        with torch.cuda.stream(self.copy_stream):
            host.copy_(coords, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(self.copy_stream)
        coords.record_stream(self.copy_stream)
        self.pending = (host, ev, properties)

    def _drain(self):
        if self.pending is None:
            return
        host, ev, props = self.pending
        ev.synchronize()
        self.f.write(format_frame(self.fmt, self.symbols, host.numpy(), self.cell, properties=props))
        self.frames += 1
        self.pending = None

    def close(self):
        self._drain()
        self.f.close()


def save_restart(path: str, species, coordinates, velocities, simulation_time_ps: float, cell=None):
    """A restart pickle with the keys of the reference's restart files."""
    data = {"nat": int(np.asarray(species).shape[0]), "nbeads": 0, "nreplicas": 0,
            "species": np.asarray(species), "coordinates": np.asarray(coordinates, np.float64),
            "vel": np.asarray(velocities, np.float64), "simulation_time_ps": float(simulation_time_ps)}
    if cell is not None:
        data["cells"] = np.asarray(cell, np.float64).reshape(1, 3, 3)
    with open(path, "wb") as f:
        pickle.dump(data, f)


def load_restart(path: str, species=None) -> Dict:
    """Read a restart pickle; ``species`` (optional) must match the file's."""
    with open(path, "rb") as f:
        data = pickle.load(f)
    if species is not None and not np.array_equal(np.asarray(data["species"]), np.asarray(species)):
        raise ValueError("restart file does not match the system's species")
    return data
