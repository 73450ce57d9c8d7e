"""Continuous-batching request loop for energy/force and MD-continuation
requests of uneven sizes on one GPU.

Two lanes share the device, each on its own CUDA stream, so their work
overlaps:

* the **single-point lane** evaluates, in one batch, every request waiting at
  the moment it is free: energy/force requests finish there, and MD requests
  get the forces at their starting positions there before they join the MD
  lane;
* the **MD lane** advances all running MD requests together in segments of
  ``segment_steps`` steps.  A segment is ``segment_steps`` repetitions of
  (integrator -> neighbour-list update when an atom moved more than half the
  skin -> energies and forces) per step, over positions, velocities and lists
  that stay on the device.  At each segment boundary finished requests leave
  and waiting ones join (continuous batching).  The first segment after a
  membership change is launched kernel by kernel; later segments of the same
  membership replay a graph captured once for it.

Requests are admitted in arrival order while the device bytes of the batches
in flight stay under the HBM budget and a lane's atom limit.  Each system's
result does not depend on which other systems share its batch: rows are
evaluated independently, the energy sum has a fixed order per system, and the
Langevin noise of a system comes from its own counter-based stream
(``fennol_md_step_systems``).  Force sums use float atomics, so forces agree
to float32 rounding rather than bitwise.

The reference has no serving loop; its MD driver (``src/fennol/md/dynamic.py``)
integrates one system with ``integrate.py:570-600``, which the MD lane
follows for every system of the batch.
"""

from __future__ import annotations

import dataclasses
import math
import time
from collections import deque
from typing import Deque, Dict, List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import call
from .md import KB_KCALMOL, MASS_DA_TO_MD, launch_flagged_rebuild
from .params import atomic_masses
from .potential import (MAX_ROW, ANIPotential, BatchLayout, GraphBuffers, HARTREE_TO_KCALMOL,
                        Workspace, _ptr, min_image_ok)


@dataclasses.dataclass
class ServeRequest:
    """One request: ``kind`` "ef" (energy and forces) or "md" (``md_steps``
    steps from ``coordinates`` and ``velocities``; Maxwell-Boltzmann
    velocities at the lane temperature drawn from ``seed`` when None)."""

    rid: int
    kind: str
    species: np.ndarray
    coordinates: np.ndarray
    cell: Optional[np.ndarray] = None
    md_steps: int = 0
    velocities: Optional[np.ndarray] = None
    seed: int = 0
    arrival: float = 0.0

    @property
    def natoms(self) -> int:
        return int(np.asarray(self.species).shape[0])


@dataclasses.dataclass
class ServeResult:
    rid: int
    kind: str
    natoms: int
    energy: float                      # model unit (Hartree), float64 sum
    forces: Optional[np.ndarray]       # model unit / A, float32 [n, 3] (ef)
    coordinates: Optional[np.ndarray]  # A, float64 (md: final positions)
    velocities: Optional[np.ndarray]   # A/ps, float64 (md: final velocities)
    arrival: float
    done: float
    error: Optional[str] = None        # set when the request was refused (no other field is valid)

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def _min_image_ok(cell: Optional[np.ndarray], reach: float) -> bool:
    return min_image_ok(cell, reach)


def _pinned(shape, dtype) -> torch.Tensor:
    return torch.empty(shape, dtype=dtype, pin_memory=True)


class _Batch:
    """Host and device data of a set of requests laid out back to back."""

    def __init__(self, pot: ANIPotential, reqs: Sequence[ServeRequest], reach: float, device):
        self.reqs = list(reqs)
        self.natoms = [r.natoms for r in reqs]
        self.offsets = np.concatenate([[0], np.cumsum(self.natoms)]).astype(np.int64)
        self.n = int(self.offsets[-1])
        species = np.concatenate([np.asarray(r.species) for r in reqs]).astype(np.int32)
        self.species = species
        cells = [None if r.cell is None else np.asarray(r.cell, np.float32).reshape(3, 3) for r in reqs]
        mi = [_min_image_ok(c, reach) for c in cells]
        has_pbc = any(c is not None for c in cells)
        sidx = pot.aev_cfg.species_index(species)
        self.layout = BatchLayout(sidx, self.natoms, cells if has_pbc else None, mi, device)


class _EFLane:
    """Single-point energy/force batches."""

    def __init__(self, engine: "ServingEngine"):
        self.e = engine
        self.stream = torch.cuda.Stream(engine.device)
        self.inflight = None
        self.cap_hint = 0  # longest row seen so far (the reference's state["npairs"] role)

    def launch(self, reqs: List[ServeRequest]):
        e, pot = self.e, self.e.pot
        with torch.cuda.stream(self.stream):
            b = _Batch(pot, reqs, pot.aev_cfg.radial_cutoff, e.device)
            xyz = np.concatenate([np.asarray(r.coordinates, np.float32) for r in reqs]).astype(np.float32)
            h_x = torch.from_numpy(xyz).pin_memory()
            coords = h_x.to(e.device, non_blocking=True)
            cap = max(b.layout.estimate_capacity(pot.aev_cfg.radial_cutoff), self.cap_hint)
            g = GraphBuffers(b.layout, pot.aev_cfg.radial_cutoff, 0.0, cap, cap)
            ws = Workspace(pot, b.layout)
            st = self.stream.cuda_stream
            self._evaluate(b, coords, g, ws, st)
            h_e = _pinned((b.layout.nsys,), torch.float64)
            h_f = _pinned((b.n, 3), torch.float32)
            h_st = _pinned((_lib.STATUS_WORDS,), torch.int32)
            h_e.copy_(ws.energy, non_blocking=True)
            h_f.copy_(ws.forces[:b.n], non_blocking=True)
            h_st.copy_(ws.status, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(self.stream)
        self.inflight = dict(batch=b, coords=coords, g=g, ws=ws, h_e=h_e, h_f=h_f, h_st=h_st, ev=ev,
                             bytes=e.bytes_per_atom * b.n)
        e.bytes_in_flight += self.inflight["bytes"]

    def _evaluate(self, b: _Batch, coords, g: GraphBuffers, ws: Workspace, st: int):
        pot = self.e.pot
        ws.status.zero_()
        call("fennol_pack_atoms", coords.data_ptr(), b.layout.t_species.data_ptr(), b.n,
             ws.xyzs.data_ptr(), st)
        g.build(b.layout, coords, ws.status, st)
        pot.launch_forces(b.layout, g, ws, st, True)
        call("fennol_forces_finalize", ws.forces4.data_ptr(), b.n, 1.0, ws.forces.data_ptr(), st)

    def poll(self, now_fn) -> bool:
        fl = self.inflight
        if fl is None or not fl["ev"].query():
            return False
        e, pot = self.e, self.e.pot
        b, ws, g = fl["batch"], fl["ws"], fl["g"]
        st = fl["h_st"].numpy()
        if st[_lib.ST_ANG_OVERFLOW]:
            raise RuntimeError(f"more than {_lib.MAX_ANGULAR_NEIGHBORS} angular neighbours around one atom")
        if st[_lib.ST_NBR_OVERFLOW]:
            # rerun the same batch with rows long enough (rare: the estimate has a margin)
            cap = (int(1.05 * st[_lib.ST_NBR_MAXCOUNT]) + 8 + 7) // 8 * 8
            if cap > MAX_ROW:
                raise RuntimeError(f"neighbour rows longer than {MAX_ROW} are not supported")
            self.cap_hint = max(self.cap_hint, cap)
            with torch.cuda.stream(self.stream):
                g2 = GraphBuffers(b.layout, pot.aev_cfg.radial_cutoff, 0.0, cap, cap)
                self._evaluate(b, fl["coords"], g2, ws, self.stream.cuda_stream)
                fl["h_e"].copy_(ws.energy, non_blocking=True)
                fl["h_f"].copy_(ws.forces[:b.n], non_blocking=True)
                fl["h_st"].copy_(ws.status, non_blocking=True)
                fl["g"] = g2
                fl["ev"].record(self.stream)
            return True
        t = now_fn()
        energies = fl["h_e"].numpy().copy()
        forces = fl["h_f"].numpy()
        to_md = []
        with torch.cuda.stream(self.stream):
            for k, r in enumerate(b.reqs):
                lo, hi = int(b.offsets[k]), int(b.offsets[k + 1])
                if r.kind == "ef":
                    e.results.append(ServeResult(r.rid, "ef", r.natoms, float(energies[k]),
                                                 forces[lo:hi].copy(), None, None, r.arrival, t))
                else:
                    to_md.append((r, ws.forces4[lo:hi].clone(), float(energies[k])))
            if to_md:
                # the MD lane reads these forces on its own stream after this event
                e.md.ready_event = torch.cuda.Event()
                e.md.ready_event.record(self.stream)
                e.md.ready.extend(to_md)
        e.bytes_in_flight -= fl["bytes"]
        self.inflight = None
        return True


class _MDLane:
    """Running MD requests advanced together, one graph replay per segment."""

    def __init__(self, engine: "ServingEngine"):
        self.e = engine
        self.stream = torch.cuda.Stream(engine.device)
        self.body_stream = torch.cuda.Stream(engine.device)  # conditional rebuild bodies
        self.members: List[dict] = []
        self.ready: List[tuple] = []
        self.ready_event: Optional[torch.cuda.Event] = None
        self.state = None
        self.inflight = None
        self.graphs: Dict[int, torch.cuda.CUDAGraph] = {}
        self.cap_hint = (0, 0)  # longest skin / radial rows seen so far
        self.captures = 0

    # ---------------------------------------------------------------- state
    def _new_state(self, keep: List[dict], new: List[tuple], b: Optional[_Batch] = None):
        """Device arrays of the next membership: continuing members' slices
        of the current arrays followed by the new members (``b``: the batch
        layout of that membership when it was prepared ahead)."""
        e, pot, dev = self.e, self.e.pot, self.e.device
        reqs = [m["req"] for m in keep] + [r for r, _, _ in new]
        if b is None:
            b = _Batch(pot, reqs, pot.aev_cfg.radial_cutoff + e.skin, dev)
        old = self.state
        xs, vs, f4s, steps = [], [], [], []
        for m in keep:
            lo, hi = m["lo"], m["hi"]
            xs.append(old["x"][lo:hi])
            vs.append(old["v"][lo:hi])
            f4s.append(old["ws"].forces4[lo:hi])
            steps.append(old["sys_step"][m["slot"]:m["slot"] + 1])
        for r, f4, _ in new:
            f4.record_stream(self.stream)
            xs.append(torch.tensor(np.asarray(r.coordinates, np.float64), device=dev))
            vs.append(torch.tensor(self._velocities(r), device=dev))
            f4s.append(f4)
            steps.append(torch.zeros(1, dtype=torch.int64, device=dev))
        masses = atomic_masses(b.species)
        mass = masses * MASS_DA_TO_MD
        x = torch.cat(xs).contiguous()
        st = dict(batch=b, x=x, v=torch.cat(vs).contiguous(),
                  inv_mass=torch.tensor(1.0 / mass, dtype=torch.float64, device=dev),
                  a2=(torch.tensor(np.sqrt((1.0 - e.a1 ** 2) * e.kT / mass), dtype=torch.float64, device=dev)
                      if e.langevin else None),
                  sys_seed=torch.tensor(np.array([r.seed for r in reqs], np.uint64).view(np.int64), device=dev),
                  sys_step=torch.cat(steps).contiguous(),
                  coords=x.to(torch.float32), x_ref=x.clone(),
                  flag=torch.zeros(1, dtype=torch.int32, device=dev))
        rc = pot.aev_cfg.radial_cutoff
        cap = max(b.layout.estimate_capacity(rc + e.skin), self.cap_hint[0])
        capr = max(b.layout.estimate_capacity(rc), self.cap_hint[1])
        st["g"] = GraphBuffers(b.layout, rc, e.skin, cap, capr)
        st["ws"] = Workspace(pot, b.layout)
        st["ws"].forces4[:b.n].copy_(torch.cat(f4s))
        members = []
        for k, r in enumerate(reqs):
            prev = keep[k] if k < len(keep) else None
            members.append(dict(req=r, lo=int(b.offsets[k]), hi=int(b.offsets[k + 1]), slot=k,
                                done=prev["done"] if prev else 0))
        return st, members

    def _velocities(self, r: ServeRequest) -> np.ndarray:
        if r.velocities is not None:
            return np.asarray(r.velocities, np.float64)
        mass = atomic_masses(r.species) * MASS_DA_TO_MD
        rng = np.random.default_rng(r.seed)
        return rng.standard_normal((r.natoms, 3)) * np.sqrt(self.e.kT / mass)[:, None]

    def _build(self, st):
        """Full list build at the current positions, enqueued without waiting:
        a row overflow shows in the status words read at the end of the
        segment, which then rolls back, regrows and runs again."""
        b = st["batch"]
        s = self.stream.cuda_stream
        st["g"].build(b.layout, st["coords"], st["ws"].status, s)
        st["g"].filter(b.layout, st["coords"], st["ws"].status, s)
        st["x_ref"].copy_(st["x"])
        st["flag"].zero_()
        call("fennol_pack_atoms", st["coords"].data_ptr(), b.layout.t_species.data_ptr(), b.n,
             st["ws"].xyzs.data_ptr(), s)

    def _launch_step(self, st, s: int):
        e, pot, b = self.e, self.e.pot, st["batch"]
        lay, g, ws = b.layout, st["g"], st["ws"]
        call("fennol_md_step_systems", b.n, lay.nsys, e.dt, st["x"].data_ptr(), st["v"].data_ptr(),
             st["inv_mass"].data_ptr(), ws.forces4.data_ptr(), e.force_scale, e.a1, _ptr(st["a2"]),
             lay.t_atom_sys.data_ptr(), lay.t_sys_start.data_ptr(), st["sys_seed"].data_ptr(),
             st["sys_step"].data_ptr(), st["coords"].data_ptr(), lay.t_species.data_ptr(),
             ws.xyzs.data_ptr(), st["x_ref"].data_ptr(), 0.5 * e.skin, st["flag"].data_ptr(), s)
        launch_flagged_rebuild(g, lay, st["coords"], ws.status, st["flag"], st["x"], st["x_ref"], s,
                               self.body_stream.cuda_stream)
        g.filter(lay, st["coords"], ws.status, s)
        pot.launch_forces(lay, g, ws, s, True)

    # ------------------------------------------------------------ segments
    def plan_next(self):
        """While a segment runs on the device, lay out the next membership on
        the host: the members that will still be running after it and the MD
        requests ready now.  Requests that become ready later join one
        segment after."""
        e, fl = self.e, self.inflight
        if fl is None:
            return
        k = fl["k"]
        keep = [m for m in self.members if m["done"] + k < m["req"].md_steps]
        admit = e._md_admits(sum(m["hi"] - m["lo"] for m in keep), pop=False)
        self.prepared = None
        if len(keep) == len(self.members) and not admit:
            return  # unchanged membership: nothing to lay out
        reqs = [m["req"] for m in keep] + [r for r, _, _ in admit]
        if not reqs:
            return
        b = _Batch(e.pot, reqs, e.pot.aev_cfg.radial_cutoff + e.skin, e.device)
        self.prepared = dict(keep=[m["req"] for m in keep], admit=list(admit), batch=b)

    def take_prepared(self) -> Optional[tuple]:
        """(admit, batch) of the prepared membership if it still applies, the
        admitted requests removed from the ready list."""
        p, self.prepared = getattr(self, "prepared", None), None
        if p is None:
            return None
        keep = [m["req"] for m in self.members if m["done"] < m["req"].md_steps]
        n = len(p["admit"])
        if len(keep) != len(p["keep"]) or any(a is not b for a, b in zip(keep, p["keep"])):
            return None
        if len(self.ready) < n or any(a is not b for a, b in zip(self.ready[:n], p["admit"])):
            return None
        del self.ready[:n]
        return p["admit"], p["batch"]

    def start_segment(self, admit: List[tuple], batch: Optional[_Batch] = None) -> bool:
        """Retire finished members, admit new ones, enqueue the next segment.
        A segment right after a membership change is launched directly; later
        segments of the same membership replay a captured CUDA graph."""
        e = self.e
        keep = [m for m in self.members if m["done"] < m["req"].md_steps]
        changed = len(keep) != len(self.members) or bool(admit) or self.state is None
        with torch.cuda.stream(self.stream):
            if admit and self.ready_event is not None:
                self.stream.wait_event(self.ready_event)
            if self.state is not None:
                self.state["ws"].status.zero_()
            if changed:
                if self.state is not None:
                    e.bytes_in_flight -= self.state["bytes"]
                self.graphs.clear()
                if not keep and not admit:
                    self.members, self.state = [], None
                    return False
                st, members = self._new_state(keep, admit, batch)
                st["bytes"] = e.bytes_per_atom_md * st["batch"].n
                e.bytes_in_flight += st["bytes"]
                self.state, self.members = st, members
                self._build(st)
            st = self.state
            k = min(e.segment_steps, min(m["req"].md_steps - m["done"] for m in self.members))
            snap = (st["x"].clone(), st["v"].clone(), st["ws"].forces4.clone(), st["sys_step"].clone())
            self._run(k, eager=changed)
            h_st = _pinned((_lib.STATUS_WORDS,), torch.int32)
            h_st.copy_(st["ws"].status, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(self.stream)
        self.inflight = dict(k=k, ev=ev, h_st=h_st, snap=snap)
        return True

    def _run(self, k: int, eager: bool):
        s = self.stream.cuda_stream
        if eager:
            for _ in range(k):
                self._launch_step(self.state, s)
            return
        if k not in self.graphs:
            graph = torch.cuda.CUDAGraph()
            graph.capture_begin()
            try:
                for _ in range(k):
                    self._launch_step(self.state, s)
            finally:
                graph.capture_end()
            self.graphs[k] = graph
            self.captures += 1
        self.graphs[k].replay()

    def poll(self, now_fn) -> bool:
        fl = self.inflight
        if fl is None or not fl["ev"].query():
            return False
        e, st = self.e, self.state
        stat = fl["h_st"].numpy()
        if stat[_lib.ST_ANG_OVERFLOW]:
            raise RuntimeError(f"more than {_lib.MAX_ANGULAR_NEIGHBORS} angular neighbours around one atom")
        if stat[_lib.ST_NBR_OVERFLOW] or stat[_lib.ST_FILTER_OVERFLOW]:
            # roll the segment back, regrow the lists, replay
            grow = e.pot.check_status(st["ws"], st["g"])
            with torch.cuda.stream(self.stream):
                x, v, f4, steps = fl["snap"]
                st["x"].copy_(x)
                st["v"].copy_(v)
                st["ws"].forces4.copy_(f4)
                st["sys_step"].copy_(steps)
                st["coords"].copy_(st["x"].to(torch.float32))
                st["g"] = GraphBuffers(st["batch"].layout, st["g"].cutoff, e.skin, *grow)
                self.cap_hint = (max(self.cap_hint[0], grow[0]), max(self.cap_hint[1], grow[1]))
                self.graphs.clear()
                st["ws"].status.zero_()
                self._build(st)
                self._run(fl["k"], eager=True)
                fl["h_st"].copy_(st["ws"].status, non_blocking=True)
                fl["ev"].record(self.stream)
            return True
        for m in self.members:
            m["done"] += fl["k"]
        finished = [m for m in self.members if m["done"] >= m["req"].md_steps]
        if finished:
            with torch.cuda.stream(self.stream):
                h_x = st["x"].cpu()
                h_v = st["v"].cpu()
                h_e = st["ws"].energy.cpu()
            t = now_fn()
            for m in finished:
                r = m["req"]
                e.results.append(ServeResult(r.rid, "md", r.natoms, float(h_e[m["slot"]]), None,
                                             h_x[m["lo"]:m["hi"]].numpy().copy(),
                                             h_v[m["lo"]:m["hi"]].numpy().copy(), r.arrival, t))
        self.inflight = None
        return True


class ServingEngine:
    """Continuous batching of energy/force and MD-continuation requests.

    ``hbm_budget_gb``: device bytes the batches in flight may hold;
    ``max_ef_atoms`` / ``max_md_atoms``: atoms per single-point batch and in
    the MD lane (latency bound).  MD uses Langevin dynamics at
    ``temperature`` with friction ``gamma_ps`` (``thermostat="NVE"`` for
    none), ``dt_fs`` steps and a ``skin`` (A) neighbour list.
    """

    def __init__(self, pot: ANIPotential, hbm_budget_gb: float = 120.0, max_ef_atoms: int = 65536,
                 max_md_atoms: int = 262144, segment_steps: int = 10, dt_fs: float = 0.5,
                 thermostat: str = "LGV", temperature: float = 300.0, gamma_ps: float = 1.0,
                 skin: float = 1.0):
        self.pot = pot
        self.device = pot.device
        self.budget = int(hbm_budget_gb * 1e9)
        self.max_ef_atoms, self.max_md_atoms = max_ef_atoms, max_md_atoms
        self.segment_steps = segment_steps
        self.dt = dt_fs / 1000.0
        self.skin = skin
        self.kT = KB_KCALMOL * temperature
        self.langevin = thermostat.upper() in ("LGV", "LANGEVIN")
        self.a1 = math.exp(-gamma_ps * self.dt) if self.langevin else 1.0
        self.force_scale = HARTREE_TO_KCALMOL / pot.unit_scale
        d0 = pot.mlp.dims[0]
        act = 2 * 2 if pot.precision != _lib.MLP_FP32 else 4
        # AEV rows (hi+lo or fp32) + dE/dAEV + neighbour rows + per-atom state
        self.bytes_per_atom = d0 * (act + 4) + 8 * 128 + 256
        self.bytes_per_atom_md = self.bytes_per_atom + 8 * 96 + 128
        self.bytes_in_flight = 0
        self.results: List[ServeResult] = []
        self.ef = _EFLane(self)
        self.md = _MDLane(self)

    def _md_admits(self, running: int, pop: bool) -> List[tuple]:
        """Ready MD requests, in order, that fit beside ``running`` atoms in
        the MD lane's atom limit and in the HBM budget (the bytes of the
        lane's current arrays are replaced by the next membership)."""
        md = self.md
        room = self.max_md_atoms - running
        other = self.bytes_in_flight - (md.state["bytes"] if md.state else 0)
        admit, atoms = [], running
        for item in list(md.ready):
            n_new = item[0].natoms
            fits = n_new <= room and other + self.bytes_per_atom_md * (atoms + n_new) <= self.budget
            if not fits and (admit or running or other):
                break
            admit.append(item)
            room -= n_new
            atoms += n_new
        if pop:
            del md.ready[:len(admit)]
        return admit

    def _take(self, queue: Deque[ServeRequest], max_atoms: int, per_atom: int) -> List[ServeRequest]:
        out, atoms = [], 0
        while queue:
            r = queue[0]
            if out and atoms + r.natoms > max_atoms:
                break
            if self.bytes_in_flight + per_atom * (atoms + r.natoms) > self.budget and (out or self.bytes_in_flight):
                break
            out.append(queue.popleft())
            atoms += r.natoms
        return out

    def run(self, requests: Sequence[ServeRequest], realtime: bool = True,
            timeout_s: float = 600.0) -> List[ServeResult]:
        """Serve ``requests`` (sorted by ``arrival``, seconds).  With
        ``realtime`` a request becomes visible when the wall clock passes its
        arrival; otherwise all are visible at once.  Returns results in
        completion order; latencies are measured on the host clock."""
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        waiting: Deque[ServeRequest] = deque()
        self.results = []
        t0 = time.perf_counter()

        def now():
            return time.perf_counter() - t0

        if not realtime:
            for r in pending:
                r.arrival = 0.0
        n_total = len(pending)
        while len(self.results) < n_total:
            t = now()
            if t > timeout_s:
                raise TimeoutError("serving loop did not finish")
            while pending and (not realtime or pending[0].arrival <= t):
                r = pending.popleft()
                if not np.all(np.isfinite(np.asarray(r.coordinates, dtype=np.float64))):
                    # refused before admission, like a host-side input check
                    self.results.append(ServeResult(r.rid, r.kind, r.natoms, float("nan"), None, None, None,
                                                    r.arrival, now(), error="non-finite coordinates"))
                    continue
                waiting.append(r)
            progressed = self.ef.poll(now)
            progressed |= self.md.poll(now)
            if self.ef.inflight is None and waiting:
                batch = self._take(waiting, self.max_ef_atoms, self.bytes_per_atom)
                if batch:
                    self.ef.launch(batch)
                    progressed = True
            if self.md.inflight is None and (self.md.members or self.md.ready):
                prepared = self.md.take_prepared()
                if prepared is not None:
                    progressed |= self.md.start_segment(*prepared)
                else:
                    running = sum(m["hi"] - m["lo"] for m in self.md.members
                                  if m["done"] < m["req"].md_steps)
                    progressed |= self.md.start_segment(self._md_admits(running, pop=True))
                if self.md.inflight is not None:
                    self.md.plan_next()
            if not progressed:
                time.sleep(2e-5)
        torch.cuda.synchronize(self.device)
        return self.results


def latency_percentiles(results: Sequence[ServeResult]) -> Dict[str, float]:
    lat = np.array([r.latency for r in results]) * 1e3
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean())}


def atom_steps(results: Sequence[ServeResult], reqs: Dict[int, ServeRequest]) -> int:
    """Energy/force evaluations done for the results: atoms for a single
    point, atoms x (steps + 1) for an MD request (its first evaluation
    included)."""
    total = 0
    for r in results:
        if r.error is not None:
            continue
        q = reqs[r.rid]
        total += r.natoms * (1 + (q.md_steps if q.kind == "md" else 0))
    return total


def serve_requests_from_stream(stream, seed: int = 0) -> List[ServeRequest]:
    """ServeRequests from :func:`fennol_b200.systems.request_stream` items
    (per-request seeds ``seed + rid`` for velocities and Langevin noise)."""
    out = []
    for rid, q in enumerate(stream):
        s = q.system
        out.append(ServeRequest(rid, q.kind, s.species, s.coordinates, s.cell, q.md_steps,
                                None, seed + rid, q.arrival_s))
    return out
