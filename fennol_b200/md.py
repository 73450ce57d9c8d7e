"""Device-resident molecular dynamics with the ANI potential.

Mirrors FeNNol's MD step (``src/fennol/md/integrate.py:570-600``):
``integrate`` (B-A-O-A, ``:286-294``) -> ``update_graphs`` (full rebuild or
skin update, ``:515-566``) -> ``update_observables`` (energy and forces,
``:298-397``).  Differences by design:

* positions and velocities are float64 on the device (the reference keeps
  the precision of ``fprec``); forces come from the float32/BF16 kernels;
* the neighbour list is rebuilt when an atom moved more than half the skin
  since the last rebuild (``trigger="displacement"``: a device flag, the
  rebuild a conditional node of the step graph), or every ``nblist_stride``
  steps like the reference (``integrate.py:498-510``) when
  ``trigger="stride"``.  In stride mode every step between rebuilds also
  checks the displacements on the device; a chunk in which an atom moved more
  than half the skin is rolled back and replayed with a shorter stride, so
  no kept step ran on a stale list (the reference trusts its stride);
* every step is captured once in a CUDA graph and replayed; capacity
  overflow (the reference's ``check_reallocate``) is detected from the device
  status words every ``check_every`` steps and answered by restoring the last
  snapshot, regrowing the lists and replaying.

Units: Angstrom, ps, kcal/mol (``md/utils.py:9``); masses follow the
reference's conversion ``mass_Da / us.DA`` (``md/initial.py:79-108``).
"""

from __future__ import annotations

import math
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._lib import ERR_UNSUPPORTED, FennolError, call, load
from .params import atomic_masses
from .potential import ANIPotential, GraphBuffers, HARTREE_TO_KCALMOL, _ptr

# atomic-unit constants of src/fennol/utils/atomic_units.py
_MPROT = 1836.1526734252586
_ANGSTROM = 0.52917721
_FS = 2.4188843e-2
_PS = _FS / 1000.0
_K_B = 3.166811563e-6
_KCALPERMOL = 627.5096080305927
MASS_DA_TO_MD = _MPROT * _KCALPERMOL * _PS ** 2 / _ANGSTROM ** 2   # Da -> kcal/mol ps^2 / A^2
KB_KCALMOL = _K_B * _KCALPERMOL                                    # kcal/mol/K


# number of rebuilds captured as conditional graph nodes (diagnostics, tests)
conditional_captures = 0


def launch_flagged_rebuild(g: GraphBuffers, layout, coords, status, flag, x, x_ref, stream: int,
                           body_stream: int):
    """Enqueue the displacement-triggered list rebuild (build, then x_ref = x
    and flag = 0).  While ``stream`` is being captured the rebuild becomes the
    body of a conditional node (captured on ``body_stream``) that a replay runs
    only when the device flag is set; uncaptured, the rebuild kernels read the
    flag and return at once when it is clear."""
    global conditional_captures
    rc = load().fennol_capture_if_begin(stream, flag.data_ptr(), body_stream)
    if rc == ERR_UNSUPPORTED:  # not capturing
        body_stream = stream
    elif rc != 0:
        raise FennolError("fennol_capture_if_begin", rc)
    else:
        conditional_captures += 1
    try:
        g.build(layout, coords, status, body_stream, enable_flag=flag)
        call("fennol_md_mark_rebuilt", layout.n, x.data_ptr(), x_ref.data_ptr(), flag.data_ptr(), body_stream)
    finally:
        if body_stream != stream:
            call("fennol_capture_if_end", body_stream)


class MDEngine:
    """Langevin (BAOAB) or NVE dynamics of one batch layout on one GPU."""

    def __init__(self, pot: ANIPotential, coordinates, species, cell=None, natoms=None,
                 dt_fs: float = 0.5, thermostat: str = "LGV", temperature: float = 300.0,
                 gamma_ps: float = 1.0, skin: float = 1.0, trigger: str = "displacement",
                 nblist_stride: Optional[int] = None, seed: int = 0, velocities=None,
                 check_every: int = 50):
        self.pot = pot
        dev = pot.device
        self.device = dev
        species = np.asarray(species)
        self.species = species
        self.cell = None if cell is None else np.asarray(cell, dtype=np.float64)
        coordinates = np.asarray(coordinates, dtype=np.float64)
        if not np.all(np.isfinite(coordinates)):
            raise ValueError("coordinates hold a NaN or an infinity")
        natoms = [species.shape[0]] if natoms is None else list(natoms)
        cells = None if cell is None else np.asarray(cell).reshape(-1, 3, 3)
        self.layout = pot.layout(species, natoms, cells, reach=pot.aev_cfg.radial_cutoff + float(skin))
        self.n = self.layout.n
        self.dt = dt_fs / 1000.0
        self.skin = float(skin)
        self.trigger = trigger
        if nblist_stride is None:
            # integrate.py:498-507: 2 A of skin lasts 40 fs at 300 K
            nblist_stride = max(1, int(math.floor(self.skin / 2.0 * 40.0 / dt_fs))) if skin > 0 else 1
        self.nblist_stride = nblist_stride
        self.stride_reductions = 0
        self.verify_stride = trigger == "stride" and self.skin > 0
        self.check_every = check_every
        mass_da = atomic_masses(species)
        mass = mass_da * MASS_DA_TO_MD
        self.mass = mass
        kT = KB_KCALMOL * temperature
        self.kT = kT
        rng = np.random.default_rng(seed)
        if velocities is None:
            v = rng.standard_normal((self.n, 3)) * np.sqrt(kT / mass)[:, None]
            if thermostat.upper() == "NVE":
                # rescale to the target temperature (thermostats.py:172-184)
                kTsys = np.sum(mass[:, None] * v ** 2) / (self.n * 3)
                v *= np.sqrt(kT / kTsys)
        else:
            v = np.asarray(velocities, dtype=np.float64)
        self.thermostat = thermostat.upper()
        if self.thermostat in ("LGV", "LANGEVIN"):
            self.a1 = math.exp(-gamma_ps * self.dt)
            a2 = np.sqrt((1.0 - self.a1 ** 2) * kT / mass)
            self.a2 = torch.tensor(a2, dtype=torch.float64, device=dev)
        elif self.thermostat in ("NVE", "NONE"):
            self.a1, self.a2 = 1.0, None
        else:
            raise ValueError(f"thermostat {thermostat} not supported on this path")
        self.seed = int(rng.integers(1 << 62))
        self.x = torch.tensor(coordinates, dtype=torch.float64, device=dev)
        self.v = torch.tensor(v, dtype=torch.float64, device=dev)
        self.inv_mass = torch.tensor(1.0 / mass, dtype=torch.float64, device=dev)
        self.x_ref = self.x.clone()
        self.coords = self.x.to(torch.float32).contiguous()
        self.flag = torch.zeros(1, dtype=torch.int32, device=dev)
        self.step_counter = torch.zeros(1, dtype=torch.int64, device=dev)
        self.step_count = 0
        self.force_scale = HARTREE_TO_KCALMOL / pot.unit_scale
        self.graph_buf, self.ws = pot.buffers(self.layout, skin=self.skin)
        self._graphs = {}
        # captures the rebuild kernels into the body of the step graph's IF node
        self._body_stream = torch.cuda.Stream(dev)
        self._snapshot = None
        self.rebuilds = 0
        self._initial_forces()

    # ------------------------------------------------------------------ core
    def _stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    def _pack(self, st):
        call("fennol_pack_atoms", self.coords.data_ptr(), self.layout.t_species.data_ptr(), self.n,
             self.ws.xyzs.data_ptr(), st)

    def _initial_forces(self):
        """Full build + forces at the initial positions (regrowing on overflow)."""
        st = self._stream()
        for _ in range(5):
            self.ws.status.zero_()
            self._pack(st)
            self.graph_buf.build(self.layout, self.coords, self.ws.status, st)
            self.graph_buf.filter(self.layout, self.coords, self.ws.status, st)
            self.pot.launch_forces(self.layout, self.graph_buf, self.ws, st, True)
            grow = self.pot.check_status(self.ws, self.graph_buf)
            if grow is None:
                break
            self.graph_buf = self.graph_buf.regrown(self.layout, *grow)
        else:
            raise RuntimeError("neighbour capacity did not converge")
        self.x_ref.copy_(self.x)
        self.flag.zero_()
        self.ws.status.zero_()

    def _launch_step(self, st, rebuild: Optional[bool]):
        """Enqueue one MD step.  rebuild: True/False (stride mode) or None
        (device displacement trigger).  Under graph capture the displacement
        rebuild is the body of a conditional node that runs only when the flag
        is set; otherwise the rebuild kernels read the flag and return at once
        when it is clear."""
        g, ws, lay = self.graph_buf, self.ws, self.layout
        use_flag = rebuild is None
        check = use_flag or (self.verify_stride and not rebuild)
        call("fennol_md_step", self.n, self.dt, self.x.data_ptr(), self.v.data_ptr(),
             self.inv_mass.data_ptr(), ws.forces4.data_ptr(), self.force_scale, self.a1,
             _ptr(self.a2), self.seed, self.step_counter.data_ptr(),
             self.coords.data_ptr(), lay.t_species.data_ptr(), ws.xyzs.data_ptr(),
             self.x_ref.data_ptr() if check else None, 0.5 * self.skin,
             self.flag.data_ptr() if check else None, st)
        if use_flag:
            launch_flagged_rebuild(g, lay, self.coords, ws.status, self.flag, self.x, self.x_ref, st,
                                   self._body_stream.cuda_stream)
        elif rebuild:
            g.build(lay, self.coords, ws.status, st)
            if self.verify_stride:
                self.x_ref.copy_(self.x)  # the stream is torch's current one (captured or not)
        g.filter(lay, self.coords, ws.status, st)
        # the finite check runs once per chunk (run), not every step
        self.pot.launch_forces(lay, g, ws, st, True, check_finite=False)

    def launches_per_step(self) -> int:
        """Kernels of this library that one graph-replayed step without a
        rebuild runs (displacement trigger: the flag-to-condition kernel; the
        rebuild kernels are in the conditional body, see rebuild_launches)."""
        n = 2  # md step + counter
        if self.trigger == "displacement":
            n += 1
        n += 1 if self.skin > 0 else 0
        n += 1 + self.pot.mlp_launches() + 1 + 1  # aev fwd, mlp, energy sum, aev bwd
        return n

    def rebuild_launches(self) -> int:
        """Kernels a rebuild adds to a step: prepare/scan/scatter/sort cells/
        cells/allpairs (+ mark/clear with the displacement trigger)."""
        return (6 if self.graph_buf.ncells > 0 else 2) + (2 if self.trigger == "displacement" else 0)

    def graph_for_step(self, k: int):
        """The one-step graph of the k-th step from now."""
        if self.trigger == "displacement":
            return self._graph_for(None, 1)
        return self._graph_for((self.step_count + k) % self.nblist_stride == 0, 1)

    def displaced_beyond_skin(self) -> bool:
        """Stride mode: did an atom move more than half the skin since its
        list was built, in a step that did not rebuild?"""
        return self.verify_stride and bool(int(self.flag.item()))

    def shorten_stride(self):
        """Roll back to the last snapshot, rebuild there and continue with a
        shorter stride (3/4 of it)."""
        self.restore()
        self.nblist_stride = max(1, (3 * self.nblist_stride) // 4)
        self.stride_reductions += 1
        self._initial_forces_from_current()

    # ---------------------------------------------------------------- graphs
    def _graph_for(self, rebuild: Optional[bool], nsteps: int):
        key = (rebuild, nsteps)
        if key not in self._graphs:
            stream = torch.cuda.Stream(self.device)
            stream.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.stream(stream):
                # warm the launch path once outside capture (function attributes)
                pass
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph, stream=stream):
                st = torch.cuda.current_stream(self.device).cuda_stream
                for _ in range(nsteps):
                    self._launch_step(st, rebuild)
            torch.cuda.current_stream(self.device).wait_stream(stream)
            self._graphs[key] = graph
        return self._graphs[key]

    def snapshot(self):
        self._snapshot = (self.x.clone(), self.v.clone(), self.x_ref.clone(), self.step_counter.clone(),
                          self.ws.forces4.clone(), self.step_count)

    def restore(self):
        x, v, xr, sc, f4, n = self._snapshot
        self.x.copy_(x)
        self.v.copy_(v)
        self.x_ref.copy_(xr)
        self.step_counter.copy_(sc)
        self.ws.forces4.copy_(f4)
        self.step_count = n
        self.coords.copy_(self.x.to(torch.float32))

    def check_finite(self):
        """Enqueue the device check of positions, velocities and forces
        (FeNNol's MD driver checks positions and velocities for NaN every
        ``nsummary`` steps, ``md/dynamic.py:204-208, 595-597``)."""
        _lib.check_finite([self.x, self.v, self.ws.forces4[:self.n]], self.ws.status, self._stream())

    def _regrow(self):
        grow = self.pot.check_status(self.ws, self.graph_buf)
        if grow is None:
            return False
        self.graph_buf = self.graph_buf.regrown(self.layout, *grow)
        self._graphs.clear()
        self.restore()
        self._initial_forces_from_current()
        return True

    def _initial_forces_from_current(self):
        self.coords.copy_(self.x.to(torch.float32))
        self._initial_forces()

    def run(self, nsteps: int, graph_steps: int = 1, sync: bool = True):
        """Advance ``nsteps`` steps; status words are checked every
        ``check_every`` steps and an overflow rolls back to the last check."""
        done = 0
        self.snapshot()
        while done < nsteps:
            chunk = min(self.check_every, nsteps - done)
            k = 0
            while k < chunk:
                if self.trigger == "displacement":
                    m = min(graph_steps, chunk - k)
                    self._graph_for(None, m).replay()
                    k += m
                else:
                    rebuild = (self.step_count + k) % self.nblist_stride == 0
                    self._graph_for(bool(rebuild), 1).replay()
                    k += 1
            self.check_finite()
            try:
                grown = self._regrow()
            except _lib.NonFiniteError as err:
                raise ValueError(f"dynamics crashed at step {self.step_count + chunk}.") from err
            if grown:
                continue  # replay the chunk with larger lists
            if self.displaced_beyond_skin():
                self.shorten_stride()
                continue  # replay the chunk with more frequent rebuilds
            self.step_count += chunk
            done += chunk
            self.snapshot()
        if sync:
            torch.cuda.synchronize(self.device)

    def run_with_frames(self, nsteps: int, every: int, frames, graph_steps: int = 1):
        """Advance ``nsteps`` steps and queue the positions every ``every``
        steps into ``frames`` (a :class:`fennol_b200.trajectory.FrameStream`);
        the copies overlap the following steps."""
        done = 0
        while done < nsteps:
            k = min(every, nsteps - done)
            self.run(k, graph_steps=graph_steps, sync=False)
            done += k
            if done % every == 0:
                frames.push(self.x, properties={"time_ps": f"{self.simulation_time_ps():.6f}"})
        torch.cuda.synchronize(self.device)

    def simulation_time_ps(self) -> float:
        return self.step_count * self.dt

    def save_restart(self, path: str):
        """Positions, velocities and time in the reference's restart layout."""
        from .trajectory import save_restart
        save_restart(path, self.species, self.x.cpu().numpy(), self.v.cpu().numpy(),
                     self.simulation_time_ps(), self.cell)

    # ------------------------------------------------------------ observables
    def potential_energy(self) -> float:
        """kcal/mol, float64 sum of the current step."""
        return float(self.ws.energy.sum()) * self.force_scale

    def kinetic_energy(self) -> float:
        out = torch.zeros(1, dtype=torch.float64, device=self.device)
        call("fennol_md_kinetic", self.n, self.v.data_ptr(), self.inv_mass.data_ptr(), out.data_ptr(),
             self._stream())
        return float(out)

    def temperature(self) -> float:
        return 2.0 * self.kinetic_energy() / (3.0 * self.n * KB_KCALMOL)

    def rebuild_count(self) -> int:
        return int(self.ws.status[_lib.ST_REBUILD_COUNT])
