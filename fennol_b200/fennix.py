"""FeNNol's model and preprocessing API over the sm_100a energy/force path.

This module mirrors the parts of FeNNol that an ANI-type model goes through,
with the same names, arguments, state dictionaries and overflow protocol, so
that code written against the reference drives the CUDA kernels unchanged:

* preprocessing classes with ``FPID``, ``init``, ``__call__(state, inputs,
  return_state_update, add_margin)``, ``process``, ``update_skin``,
  ``check_reallocate``, ``get_processor``, ``get_graph_properties``
  (``src/fennol/models/preprocessing.py:22-72, 357-367, 781-1320, 1321-1490``)
  and their chain (``:1825-1925``);
* the ``ANI_AEV`` and ``SPECIES_INDEX_NET`` module descriptions
  (``embeddings/ani.py:9-44``, ``misc/nets.py:301-330``);
* the ``FENNIX`` wrapper (``fennix.py:27-690``): construction from the
  ``modules`` / ``preprocessing`` dictionaries, ``preprocess``,
  ``total_energy``, ``energy_and_forces``, ``__call__``, ``save``/``load``
  and the ``unit`` conversion of returned energies and forces;
* registration of external preprocessing classes and modules by ``FPID`` /
  ``FID`` (``modules.py:84-91``).

Differences that follow from the B200 design, not from the reference:

* a graph is stored as per-atom neighbour rows (``nbr_j`` int32 [N, cap],
  ``nbr_shift`` packed signed-byte cell shifts, ``nbr_count``) instead of the
  padded ``edge_src``/``edge_dst`` list; :func:`graph_edges` gives the
  reference's edge-list view of the same pairs;
* the angular extension does not materialise triplets: the AEV kernels form
  the pairs of angular neighbours of each centre on chip, up to
  ``MAX_ANGULAR_NEIGHBORS`` per atom (more raises, since that limit is fixed);
* the geometry processors (``GraphProcessor``, ``GraphFilterProcessor``,
  ``GraphAngleProcessor``) are fused into the AEV kernels;
* energies, forces and embeddings are torch tensors on the CUDA device.

Every compute step runs in ``libfennol_b200.so``; there is no CPU path.
"""

from __future__ import annotations

import dataclasses
import re
import weakref
from collections import OrderedDict
from copy import deepcopy
from typing import Any, ClassVar, Dict, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from ._lib import call
from .fnx import load_model_dict, save_model_dict
from .params import (PERIODIC_TABLE, PERIODIC_TABLE_REV_IDX, AEVConfig, MLPConfig,
                     init_weights, variables_to_weights, weights_to_variables)
from .potential import MAX_ROW, ANIPotential, BatchLayout, Workspace, _ceil, _stream

# multipliers from Hartree (atomic units, fennol/utils/atomic_units.py)
ENERGY_UNITS = {
    "HA": 1.0, "HARTREE": 1.0, "AU": 1.0,
    "KCALPERMOL": 627.5096080305927,
    "EV": 27.211386024367243,
    "KJPERMOL": 2625.4996394798254,
    "MEV": 27211.386024367243,
}


def energy_multiplier(unit) -> float:
    """Hartree -> ``unit`` (a float is returned unchanged)."""
    if isinstance(unit, (int, float)):
        return float(unit)
    key = str(unit).upper().replace(" ", "").replace("_", "")
    if key not in ENERGY_UNITS:
        raise ValueError(f"unknown energy unit {unit!r}")
    return ENERGY_UNITS[key]


PREPROCESSING: Dict[str, type] = {}
MODULES: Dict[str, type] = {}


def register_preprocessing(cls):
    """Register a preprocessing class under its ``FPID``."""
    PREPROCESSING[cls.FPID.upper()] = cls
    return cls


def register_module(cls):
    """Register a module description under its ``FID``."""
    MODULES[cls.FID.upper()] = cls
    return cls


# ----------------------------------------------------------------- graphs
@dataclasses.dataclass
class NeighborRows:
    """One neighbour list on the device: ``count[i]`` valid entries in row
    ``i`` of ``j`` (neighbour index) and ``shift`` (cell shift of the
    neighbour's image, 3 signed bytes)."""

    j: torch.Tensor
    shift: torch.Tensor
    count: torch.Tensor
    cutoff: float

    @property
    def capacity(self) -> int:
        return int(self.j.shape[1])

    @classmethod
    def empty(cls, n: int, cap: int, cutoff: float, device) -> "NeighborRows":
        # the builders write every row's count and its entries below it; the
        # kernels and graph_edges read nothing past the count
        n = max(n, 1)
        return cls(torch.empty((n, cap), dtype=torch.int32, device=device),
                   torch.empty((n, cap), dtype=torch.int32, device=device),
                   torch.zeros(n, dtype=torch.int32, device=device), float(cutoff))


def _status(device) -> torch.Tensor:
    return torch.zeros(_lib.STATUS_WORDS, dtype=torch.int32, device=device)


def _grow(maxcount: int, mult: float, add: int) -> int:
    cap = _ceil(int(mult * maxcount) + add, 8)
    if cap > MAX_ROW:
        raise RuntimeError(f"neighbour rows longer than {MAX_ROW} are not supported")
    return cap


def _build_rows(layout: BatchLayout, coords: torch.Tensor, cutoff: float, cap: int,
                status: torch.Tensor) -> NeighborRows:
    grid, nrep, ncells = layout.plan(cutoff)
    rows = NeighborRows.empty(layout.n, cap, cutoff, layout.device)
    ws_bytes = _lib.load().fennol_graph_workspace_bytes(max(layout.n, 1), ncells)
    ws = torch.empty(int(ws_bytes), dtype=torch.uint8, device=layout.device)
    call("fennol_graph_build", coords.data_ptr(), layout.n, layout.t_atom_sys.data_ptr(), layout.nsys,
         layout.t_sys_start.data_ptr(), layout.t_mode.data_ptr(), layout.t_cell.data_ptr(),
         layout.t_recip.data_ptr(), grid.data_ptr(), nrep.data_ptr(), ncells, float(cutoff), cap,
         rows.j.data_ptr(), rows.shift.data_ptr(), rows.count.data_ptr(), status.data_ptr(),
         ws.data_ptr(), ws.numel(), None, _stream(layout.device))
    return rows


def _filter_rows(layout: BatchLayout, coords: torch.Tensor, parent: NeighborRows, cutoff: float,
                 cap: int, status: torch.Tensor) -> NeighborRows:
    rows = NeighborRows.empty(layout.n, cap, cutoff, layout.device)
    call("fennol_graph_filter", coords.data_ptr(), layout.n, layout.t_atom_sys.data_ptr(),
         layout.t_cell.data_ptr(), parent.j.data_ptr(), parent.shift.data_ptr(), parent.count.data_ptr(),
         parent.capacity, float(cutoff), cap, rows.j.data_ptr(), rows.shift.data_ptr(),
         rows.count.data_ptr(), status.data_ptr(), _stream(layout.device))
    return rows


class OverflowFlag:
    """A graph layer's ``overflow`` flag (the reference's boolean array): true
    when any of the given device status words is set.  Reading it (``bool``,
    ``item``) copies those words to the host; nothing is launched or read
    until then, so calls that check every status word at once never do."""

    __slots__ = ("status", "words")

    def __init__(self, status: torch.Tensor, words: Tuple[int, ...]):
        self.status, self.words = status, tuple(words)

    def item(self) -> bool:
        host = self.status.cpu()
        return any(int(host[w]) != 0 for w in self.words)

    def __bool__(self) -> bool:
        return self.item()

    def __repr__(self) -> str:
        return f"OverflowFlag({self.item()})"


def _overflow(status: torch.Tensor, *words: int) -> OverflowFlag:
    return OverflowFlag(status, words)


@register_preprocessing
@dataclasses.dataclass(frozen=True)
class GraphGenerator:
    """Periodic cell-list neighbour search (``preprocessing.py:22-696``).

    State keys: ``max_neigh`` (row length, the counterpart of ``npairs``),
    ``max_neigh_skin`` when ``nblist_skin`` is set, ``nblist_mult_size``.
    With a skin the build list (cutoff + skin) is kept under ``*_skin`` keys
    and ``update_skin`` re-filters it to the cutoff with the current
    coordinates (``:640-696``).
    """

    cutoff: float
    graph_key: str = "graph"
    switch_params: dict = dataclasses.field(default_factory=dict)
    kmax: int = 30
    kthr: float = 1e-6
    k_space: bool = False
    mult_size: float = 1.05
    add_neigh: int = 8

    FPID: ClassVar[str] = "GRAPH"

    def __post_init__(self):
        if self.k_space:
            raise NotImplementedError("k-space graph data is outside the CUDA energy path")
        _check_switch(self.switch_params)

    def init(self):
        return {"max_nat": 1, "max_neigh": 0, "nblist_mult_size": self.mult_size}

    def get_processor(self):
        return GraphProcessor, {"cutoff": self.cutoff, "graph_key": self.graph_key,
                                "switch_params": self.switch_params,
                                "name": f"{self.graph_key}_Processor"}

    def get_graph_properties(self):
        return {self.graph_key: {"cutoff": self.cutoff, "directed": True}}

    def __call__(self, state, inputs, return_state_update=False, add_margin=False):
        graph = inputs.get(self.graph_key, {})
        if "keep_graph" in graph:
            return (state, inputs, {}) if return_state_update else (state, inputs)
        layout, coords = inputs["_layout"], inputs["_coords"]
        new_state, state_up = dict(state), {}
        mult = state.get("nblist_mult_size", self.mult_size)
        if mult < 1.0:
            raise ValueError("mult_size should be larger or equal than 1.0")
        skin = float(state.get("nblist_skin", 0.0))
        rc_build = self.cutoff + skin
        cap_prev = int(state.get("max_neigh", 0))
        cap = cap_prev or layout.estimate_capacity(rc_build)
        if add_margin:
            cap = _grow(cap, mult, self.add_neigh)
        status = _status(layout.device)
        for _ in range(8):
            status.zero_()
            rows = _build_rows(layout, coords, rc_build, cap, status)
            st = status.cpu().numpy()
            if not st[_lib.ST_NBR_OVERFLOW]:
                break
            cap = _grow(int(st[_lib.ST_NBR_MAXCOUNT]), mult, self.add_neigh)
        else:
            raise RuntimeError("neighbour capacity did not converge")
        if cap != cap_prev:
            state_up["max_neigh"] = (cap, cap_prev)
            new_state["max_neigh"] = cap
        out = {**graph, "cutoff": self.cutoff, "status": status,
               "overflow": _overflow(status, _lib.ST_NBR_OVERFLOW)}
        if skin > 0:
            capr_prev = int(state.get("max_neigh_skin", 0))
            capr = capr_prev or layout.estimate_capacity(self.cutoff)
            if add_margin:
                capr = _grow(capr, mult, self.add_neigh)
            for _ in range(8):
                status.zero_()
                radial = _filter_rows(layout, coords, rows, self.cutoff, capr, status)
                st = status.cpu().numpy()
                if not st[_lib.ST_FILTER_OVERFLOW]:
                    break
                capr = _grow(int(st[_lib.ST_FILTER_MAXCOUNT]), mult, self.add_neigh)
            if capr != capr_prev:
                state_up["max_neigh_skin"] = (capr, capr_prev)
                new_state["max_neigh_skin"] = capr
            out.update(rows=radial, rows_skin=rows, skin=skin,
                       overflow=_overflow(status, _lib.ST_FILTER_OVERFLOW))
        else:
            out.update(rows=rows)
        output = {**inputs, self.graph_key: out}
        return (new_state, output, state_up) if return_state_update else (new_state, output)

    def process(self, state, inputs):
        """Rebuild at the capacities in ``state``; sets ``overflow``."""
        layout, coords = inputs["_layout"], inputs["_coords"]
        graph = dict(inputs.get(self.graph_key, {}))
        skin = float(state.get("nblist_skin", 0.0))
        status = graph.get("status")
        if status is None:
            status = _status(layout.device)
        else:
            status.zero_()
        rows = _build_rows(layout, coords, self.cutoff + skin, int(state["max_neigh"]), status)
        graph.update(status=status)
        if skin > 0:
            graph["rows_skin"] = rows
            graph["rows"] = _filter_rows(layout, coords, rows, self.cutoff,
                                         int(state["max_neigh_skin"]), status)
            graph["overflow"] = _overflow(status, _lib.ST_NBR_OVERFLOW, _lib.ST_FILTER_OVERFLOW)
        else:
            graph["rows"] = rows
            graph["overflow"] = _overflow(status, _lib.ST_NBR_OVERFLOW)
        return {**inputs, self.graph_key: graph}

    def update_skin(self, inputs):
        """Re-filter the skin list to the cutoff (``preprocessing.py:640-696``)."""
        graph = dict(inputs[self.graph_key])
        if "rows_skin" not in graph:
            return inputs
        layout, coords = inputs["_layout"], inputs["_coords"]
        status = graph["status"]
        graph["rows"] = _filter_rows(layout, coords, graph["rows_skin"], self.cutoff,
                                     graph["rows"].capacity, status)
        graph["overflow"] = _overflow(status, _lib.ST_FILTER_OVERFLOW)
        return {**inputs, self.graph_key: graph}

    def check_reallocate(self, state, inputs, parent_overflow=False):
        return _check_reallocate(self, state, inputs, parent_overflow,
                                 inputs[self.graph_key].get("overflow", False))


@register_preprocessing
@dataclasses.dataclass(frozen=True)
class GraphFilter:
    """Sub-graph of a parent graph within a smaller cutoff
    (``preprocessing.py:781-960``).  State key: ``max_neigh``."""

    cutoff: float
    parent_graph: str
    graph_key: str
    remove_hydrogens: bool = False
    switch_params: dict = dataclasses.field(default_factory=dict)
    k_space: bool = False
    kmax: int = 30
    kthr: float = 1e-6
    mult_size: float = 1.05
    add_neigh: int = 8

    FPID: ClassVar[str] = "GRAPH_FILTER"

    def __post_init__(self):
        if self.k_space or self.remove_hydrogens:
            raise NotImplementedError("k-space data and hydrogen removal are outside the CUDA energy path")
        _check_switch(self.switch_params)

    def init(self):
        return {"max_neigh": 0, "nblist_mult_size": self.mult_size}

    def get_processor(self):
        return GraphFilterProcessor, {"cutoff": self.cutoff, "graph_key": self.graph_key,
                                      "parent_graph": self.parent_graph,
                                      "name": f"{self.graph_key}_Filter_{self.parent_graph}",
                                      "switch_params": self.switch_params}

    def get_graph_properties(self):
        return {self.graph_key: {"cutoff": self.cutoff, "directed": True,
                                 "parent_graph": self.parent_graph}}

    def __call__(self, state, inputs, return_state_update=False, add_margin=False):
        layout, coords = inputs["_layout"], inputs["_coords"]
        parent = inputs[self.parent_graph]
        if self.cutoff > parent["cutoff"] + 1e-6:
            raise ValueError("GraphFilter cutoff larger than the parent graph's")
        new_state, state_up = dict(state), {}
        mult = state.get("nblist_mult_size", self.mult_size)
        cap_prev = int(state.get("max_neigh", 0))
        cap = cap_prev or layout.estimate_capacity(self.cutoff)
        if add_margin:
            cap = _grow(cap, mult, self.add_neigh)
        status = _status(layout.device)
        for _ in range(8):
            status.zero_()
            rows = _filter_rows(layout, coords, parent["rows"], self.cutoff, cap, status)
            st = status.cpu().numpy()
            if not st[_lib.ST_FILTER_OVERFLOW]:
                break
            cap = _grow(int(st[_lib.ST_FILTER_MAXCOUNT]), mult, self.add_neigh)
        else:
            raise RuntimeError("filtered neighbour capacity did not converge")
        if cap != cap_prev:
            state_up["max_neigh"] = (cap, cap_prev)
            new_state["max_neigh"] = cap
        graph = {**inputs.get(self.graph_key, {}), "cutoff": self.cutoff, "rows": rows,
                 "parent_graph": self.parent_graph, "status": status,
                 "overflow": _overflow(status, _lib.ST_FILTER_OVERFLOW)}
        output = {**inputs, self.graph_key: graph}
        return (new_state, output, state_up) if return_state_update else (new_state, output)

    def process(self, state, inputs):
        layout, coords = inputs["_layout"], inputs["_coords"]
        graph = dict(inputs.get(self.graph_key, {}))
        status = graph.get("status")
        if status is None:
            status = _status(layout.device)
        else:
            status.zero_()
        graph.update(cutoff=self.cutoff, parent_graph=self.parent_graph, status=status,
                     rows=_filter_rows(layout, coords, inputs[self.parent_graph]["rows"], self.cutoff,
                                       int(state["max_neigh"]), status),
                     overflow=_overflow(status, _lib.ST_FILTER_OVERFLOW))
        return {**inputs, self.graph_key: graph}

    def update_skin(self, inputs):
        graph = inputs.get(self.graph_key)
        if graph is None or "rows" not in graph:
            return inputs
        return self.process({"max_neigh": graph["rows"].capacity}, inputs)

    def check_reallocate(self, state, inputs, parent_overflow=False):
        return _check_reallocate(self, state, inputs, parent_overflow,
                                 inputs[self.graph_key].get("overflow", False))


@register_preprocessing
@dataclasses.dataclass(frozen=True)
class GraphAngularExtension:
    """Marks a graph for angular use (``preprocessing.py:1047-1280``).

    The reference materialises every pair of edges sharing a centre
    (``angle_src``, ``angle_dst``, ``central_atom``).  Here the AEV kernels
    form those pairs on chip from each centre's neighbours, so this step
    records the fixed per-centre limit; exceeding it is reported by the AEV
    kernels and raises.
    """

    graph_key: str
    mult_size: float = 1.05
    add_neigh: int = 5

    FPID: ClassVar[str] = "GRAPH_ANGULAR_EXTENSION"

    def init(self):
        return {"max_neigh": _lib.MAX_ANGULAR_NEIGHBORS, "nblist_mult_size": self.mult_size}

    def get_processor(self):
        return GraphAngleProcessor, {"graph_key": self.graph_key,
                                     "name": f"{self.graph_key}_AngleProcessor"}

    def get_graph_properties(self):
        return {self.graph_key: {"has_angles": True}}

    def __call__(self, state, inputs, return_state_update=False, add_margin=False):
        out = self.process(state, inputs)
        return (dict(state), out, {}) if return_state_update else (dict(state), out)

    def process(self, state, inputs):
        graph = {**inputs[self.graph_key], "angles_on_chip": True,
                 "max_angular_neighbors": _lib.MAX_ANGULAR_NEIGHBORS}
        return {**inputs, self.graph_key: graph}

    def update_skin(self, inputs):
        return inputs

    def check_reallocate(self, state, inputs, parent_overflow=False):
        return state, {}, inputs, bool(parent_overflow)


@register_preprocessing
@dataclasses.dataclass(frozen=True)
class SpeciesIndexer:
    """Per-species atom index lists (``preprocessing.py:1321-1490``).

    Output as in the reference: a dict ``{symbol: int32[size]}`` padded with
    ``N``, or a dense ``[len(species_order), max_size]`` array when
    ``species_order`` is set.  The CUDA networks read the species-sorted
    128-row tiles of the batch layout instead; this index is for other
    consumers of the inputs dictionary.
    """

    output_key: str = "species_index"
    species_order: Optional[str] = None
    add_atoms: int = 0
    add_atoms_margin: int = 10

    FPID: ClassVar[str] = "SPECIES_INDEXER"

    def init(self):
        return {"sizes": {}}

    def __call__(self, state, inputs, return_state_update=False, add_margin=False):
        species = np.asarray(inputs["species"], dtype=np.int32)
        nat = species.shape[0]
        members = _species_members(inputs, species)
        new_state, state_up = dict(state), {}
        sizes = dict(state.get("sizes", {}))
        new_sizes = dict(sizes)
        grew = False
        counts_of = {s: len(m) for s, m in members.items()}
        for s, c in counts_of.items():
            if c > sizes.get(s, 0):
                grew = True
                extra = state.get("add_atoms", self.add_atoms)
                if add_margin:
                    extra += state.get("add_atoms_margin", self.add_atoms_margin)
                new_sizes[s] = c + extra
        if grew:
            state_up["sizes"] = (new_sizes, sizes)
            new_state["sizes"] = new_sizes
        if self.species_order is not None:
            order = [el.strip() for el in self.species_order.split(",")]
            max_prev = state.get("max_size", 0)
            max_size = max(new_sizes.values()) if new_sizes else 0
            if max_size > max_prev:
                state_up["max_size"] = (max_size, max_prev)
                new_state["max_size"] = max_size
            index = np.full((len(order), max_size), nat, dtype=np.int32)
            for i, el in enumerate(order):
                z = PERIODIC_TABLE_REV_IDX[el]
                if z in counts_of:
                    index[i, :counts_of[z]] = members[z]
        else:
            index = {PERIODIC_TABLE[s]: np.full(c, nat, dtype=np.int32) for s, c in new_sizes.items()}
            for s, c in counts_of.items():
                index[PERIODIC_TABLE[s]][:c] = members[s]
        output = {**inputs, self.output_key: index, self.output_key + "_overflow": False}
        return (new_state, output, state_up) if return_state_update else (new_state, output)

    def process(self, state, inputs):
        species = np.asarray(inputs["species"], dtype=np.int32)
        sizes = state.get("sizes", {})
        overflow = any(len(m) > sizes.get(s, 0) for s, m in _species_members(inputs, species).items())
        _, out = self(state, inputs)
        out[self.output_key + "_overflow"] = overflow
        return out

    def update_skin(self, inputs):
        return inputs

    def check_reallocate(self, state, inputs, parent_overflow=False):
        return _check_reallocate(self, state, inputs, parent_overflow,
                                 inputs[self.output_key + "_overflow"])


_MEMBERS: "weakref.WeakKeyDictionary[BatchLayout, Dict[int, np.ndarray]]" = weakref.WeakKeyDictionary()


def _species_members(inputs, species: np.ndarray) -> Dict[int, np.ndarray]:
    """Atom indices of each atomic number (> 0) present, ascending; kept with
    the batch layout, which changes whenever the species do."""
    layout = inputs.get("_layout")
    hit = _MEMBERS.get(layout) if layout is not None else None
    if hit is not None:
        return hit
    order = np.argsort(species, kind="stable").astype(np.int32)
    z, first = np.unique(species[order], return_index=True)
    bounds = list(first) + [len(order)]
    members = {int(v): order[bounds[k]:bounds[k + 1]] for k, v in enumerate(z) if v > 0}
    for m in members.values():
        m.flags.writeable = False
    if layout is not None:
        _MEMBERS[layout] = members
    return members


def _check_reallocate(layer, state, inputs, parent_overflow, own_overflow):
    """The reference's protocol (``preprocessing.py:357-367``): rerun the host
    build with a margin when this layer or a parent overflowed."""
    own_overflow = bool(own_overflow)
    if not (parent_overflow or own_overflow):
        return state, {}, inputs, False
    state, inputs, state_up = layer(state, inputs, return_state_update=True,
                                    add_margin=bool(own_overflow))
    return state, state_up, inputs, True


def _check_switch(switch_params):
    p = dict(switch_params or {})
    kind = str(p.pop("switch_type", "cosine")).lower()
    p.pop("cutoff", None)
    power = float(p.pop("p", 1.0))
    if kind != "cosine" or power != 1.0 or p:
        raise NotImplementedError(f"switch {switch_params}: only the cosine switch is fused "
                                  "into the AEV kernels")


class GraphProcessor:
    """Geometry of a graph (``preprocessing.py:699-777``); computed inside
    the AEV kernels from the neighbour rows, so it has no separate launch."""


class GraphFilterProcessor(GraphProcessor):
    """Geometry of a filtered graph (``preprocessing.py:963-1043``); fused."""


class GraphAngleProcessor(GraphProcessor):
    """Angles of an angular graph (``preprocessing.py:1283-1317``); fused."""


class PreprocessingChain:
    """Chain of preprocessing layers (``preprocessing.py:1825-1925``).

    ``check_input`` also builds the batch layout (systems, cells,
    species-sorted rows) that every layer and the kernels read, cached on
    species, system sizes and cells.
    """

    def __init__(self, layers: Sequence[Any], use_atom_padding: bool = False, device="cuda",
                 species_order: Sequence[str] = ()):
        if not layers:
            raise ValueError("Error: no Preprocessing layers were provided.")
        self.layers = tuple(layers)
        self.use_atom_padding = use_atom_padding
        self.device = torch.device(device)
        self.species_order = tuple(species_order)
        self._layout_key = None
        self._layout = None

    def init(self):
        return {"check_input": True, "layers_state": tuple(layer.init() for layer in self.layers)}

    def check_input(self, inputs: Dict[str, Any]) -> Dict[str, Any]:
        if "species" not in inputs or "coordinates" not in inputs:
            raise ValueError("species and coordinates must be provided")
        species = np.asarray(_host(inputs["species"]), dtype=np.int32).reshape(-1)
        nat = species.shape[0]
        natoms = np.asarray(_host(inputs.get("natoms", [nat])), dtype=np.int32).reshape(-1)
        cells = recips = None
        if "cells" in inputs:
            given = np.asarray(_host(inputs["cells"]))
            if given.ndim == 2:
                given = given[None]
            # the reciprocal cells as the reference forms them (check_input,
            # preprocessing.py:1780-1781): the caller's, or the inverse of the
            # caller's cells in their own precision; float32 in the builder (:126)
            if "reciprocal_cells" in inputs:
                recips = np.asarray(_host(inputs["reciprocal_cells"])).reshape(-1, 3, 3)
            else:
                recips = np.linalg.inv(given)
            recips = recips.astype(np.float32)
            cells = given.astype(np.float32)
        minimum_image = "minimum_image" in inputs.get("flags", {})
        # the layout (species-sorted rows, cell plans) is rebuilt only when the
        # species, system sizes, cells or image convention change; a repeated
        # system costs one comparison per array
        c = self._layout_key
        if not (c is not None and c[4] == minimum_image and _same(c[0], species)
                and _same(c[1], natoms) and _same(c[2], cells) and _same(c[3], recips)):
            if int(natoms.sum()) != nat:
                raise ValueError("natoms does not add up to the number of atoms")
            if self.species_order:
                sidx = AEVConfig(species_order=self.species_order).species_index(species)
            else:
                sidx = np.zeros(nat, np.int32)
            cl = None if cells is None else list(cells)
            self._layout = BatchLayout(sidx, natoms, cl, minimum_image, self.device, reciprocal_cells=recips)
            expected = np.repeat(np.arange(natoms.shape[0], dtype=np.int32), natoms)
            frozen = [None if a is None else a.copy() for a in (species, natoms, cells, recips)]
            for a in frozen + [expected]:
                if a is not None:
                    a.flags.writeable = False
            c = self._layout_key = (*frozen, minimum_image, expected)
        expected = c[5]
        batch_index = inputs.get("batch_index")
        if batch_index is not None and not np.array_equal(np.asarray(_host(batch_index)), expected):
            raise ValueError("atoms must be grouped by system in batch order")
        out = {**inputs, "species": c[0], "natoms": c[1], "batch_index": expected}
        if cells is not None:
            out["cells"] = c[2]
            out["reciprocal_cells"] = c[3]
        coords = torch.as_tensor(inputs["coordinates"], dtype=torch.float32)
        coords = coords.to(self.device, non_blocking=True).reshape(-1, 3).contiguous()
        out["_layout"] = self._layout
        out["_coords"] = coords
        return out

    def __call__(self, state, inputs):
        if state.get("check_input", True):
            inputs = self.check_input(inputs)
        layer_state = state["layers_state"]
        new_layer_state = []
        for i, layer in enumerate(self.layers):
            s, inputs = layer(layer_state[i], inputs, return_state_update=False)
            new_layer_state.append(s)
        return {**state, "layers_state": tuple(new_layer_state)}, inputs

    def process(self, state, inputs):
        for i, layer in enumerate(self.layers):
            inputs = layer.process(state["layers_state"][i], inputs)
        return inputs

    def update_skin(self, inputs):
        for layer in self.layers:
            inputs = layer.update_skin(inputs)
        return inputs

    def check_reallocate(self, state, inputs):
        new_state, state_up = [], []
        parent_overflow = False
        for i, layer in enumerate(self.layers):
            s, s_up, inputs, parent_overflow = layer.check_reallocate(
                state["layers_state"][i], inputs, parent_overflow)
            new_state.append(s)
            state_up.append(s_up)
        if not parent_overflow:
            return state, {}, inputs, False
        return {**state, "layers_state": tuple(new_state)}, state_up, inputs, True

    def init_with_output(self, inputs):
        return self(self.init(), inputs)

    def get_processors(self):
        return [layer.get_processor() for layer in self.layers if hasattr(layer, "get_processor")]

    def get_graphs_properties(self):
        props: Dict[str, dict] = {}
        for layer in self.layers:
            if hasattr(layer, "get_graph_properties"):
                for k, v in layer.get_graph_properties().items():
                    props[k] = {**props.get(k, {}), **v}
        return props


def _status_tensors(prepared: Dict[str, Any]) -> list:
    """The distinct device status words of the graph layers in a processed
    inputs dictionary."""
    pending, seen = [], set()
    for val in prepared.values():
        st = val.get("status") if isinstance(val, dict) else None
        if isinstance(st, torch.Tensor) and id(st) not in seen:
            seen.add(id(st))
            pending.append(st)
    return pending


def _scaled(x: torch.Tensor, fac: float) -> torch.Tensor:
    """``x * fac`` as a new tensor; ``x`` itself (already a copy owned by the
    caller) when the factor is 1."""
    return x if fac == 1.0 else x * fac


def _same(a, b) -> bool:
    if a is None or b is None:
        return a is b
    return a.shape == b.shape and np.array_equal(a, b)


def _host(x):
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy()
    return x


# ---------------------------------------------------------------- modules
@register_module
@dataclasses.dataclass(frozen=True)
class ANIAEV:
    """``ANI_AEV`` hyper-parameters (``embeddings/ani.py:9-44``); the cutoffs
    come from the graphs' properties as in the reference (``:66, :91``)."""

    _graphs_properties: dict
    species_order: Any
    graph_angle_key: str
    radial_eta: float = 16.0
    angular_eta: float = 8.0
    radial_dist_divisions: int = 16
    angular_dist_divisions: int = 4
    zeta: float = 32.0
    angle_sections: int = 4
    radial_start: float = 0.8
    angular_start: float = 0.8
    embedding_key: str = "embedding"
    graph_key: str = "graph"
    name: str = "embedding"

    FID: ClassVar[str] = "ANI_AEV"

    def species(self) -> Tuple[str, ...]:
        return _species_list(self.species_order)

    def config(self) -> AEVConfig:
        props = self._graphs_properties
        return AEVConfig(species_order=self.species(),
                         radial_cutoff=float(props[self.graph_key]["cutoff"]),
                         angular_cutoff=float(props[self.graph_angle_key]["cutoff"]),
                         radial_eta=float(self.radial_eta), angular_eta=float(self.angular_eta),
                         radial_dist_divisions=int(self.radial_dist_divisions),
                         angular_dist_divisions=int(self.angular_dist_divisions),
                         zeta=float(self.zeta), angle_sections=int(self.angle_sections),
                         radial_start=float(self.radial_start),
                         angular_start=float(self.angular_start))


@register_module
@dataclasses.dataclass(frozen=True)
class SpeciesIndexNet:
    """``SPECIES_INDEX_NET`` fields (``misc/nets.py:301-330``).  The CUDA
    networks take CELU activations, biases and three hidden layers."""

    output_dim: int
    hidden_neurons: Any
    species_order: Any = None
    activation: Any = "silu"
    use_bias: bool = True
    input_key: Optional[str] = None
    species_index_key: str = "species_index"
    output_key: Optional[str] = None
    squeeze: bool = False
    kernel_init: Any = "lecun_normal()"
    check_unhandled: bool = True
    name: str = "energy"

    FID: ClassVar[str] = "SPECIES_INDEX_NET"

    def species(self) -> Tuple[str, ...]:
        if isinstance(self.hidden_neurons, dict):
            return tuple(self.hidden_neurons.keys())
        return _species_list(self.species_order)

    def hidden(self) -> Tuple[int, ...]:
        h = self.hidden_neurons
        if isinstance(h, dict):
            sizes = {tuple(v) for v in h.values()}
            if len(sizes) != 1:
                raise NotImplementedError("per-species hidden sizes differ")
            return sizes.pop()
        return tuple(int(v) for v in h)

    def celu_alpha(self) -> float:
        return parse_celu(self.activation)

    @property
    def out_key(self) -> str:
        return self.name if self.output_key is None else self.output_key


def parse_celu(activation) -> float:
    """alpha of a CELU activation string (``"celu"``,
    ``"partial(celu,alpha=0.1)"``, ``"jax.nn.celu"``); other activations raise."""
    s = str(activation).replace(" ", "")
    m = re.fullmatch(r"(?:partial\()?(?:jax\.nn\.|nn\.)?celu(?:,alpha=([0-9.eE+-]+))?\)?", s)
    if m is None:
        raise NotImplementedError(f"activation {activation!r}: the CUDA networks fuse CELU only")
    return float(m.group(1)) if m.group(1) else 1.0


def _species_list(order) -> Tuple[str, ...]:
    if order is None:
        raise ValueError("species_order must be provided")
    if isinstance(order, str):
        return tuple(el.strip() for el in order.split(","))
    return tuple(order)


# ------------------------------------------------------------------ FENNIX
class FENNIX:
    """FeNNol's model wrapper for ANI-type models on the CUDA path
    (``fennix.py:27-690``).

    Extra keyword arguments of this implementation: ``precision`` (``"fp32"``,
    ``"bf16"``, ``"bf16x2"``, ``"bf16x3"``, see :class:`ANIPotential`),
    ``device``, and ``variables`` may also be a list of variables trees (an
    ensemble whose energies are averaged).  ``rng_key`` is an integer seed:
    weights are drawn N(0, 1/fan_in) with zero biases.
    """

    def __init__(self, cutoff: float, modules, preprocessing=OrderedDict(), example_data=None,
                 rng_key=None, variables=None, energy_terms=None, use_atom_padding: bool = False,
                 graph_config: Dict = {}, energy_unit: str = "Ha", precision: str = "bf16x2",
                 device="cuda", **kwargs):
        self._input_args = {"cutoff": cutoff, "modules": OrderedDict(deepcopy(modules)),
                            "preprocessing": OrderedDict(deepcopy(preprocessing)),
                            "energy_unit": energy_unit}
        self.energy_unit = energy_unit
        self.Ha_to_model_energy = energy_multiplier(energy_unit)
        self.cutoff = cutoff
        self.energy_terms = list(energy_terms) if energy_terms is not None else None
        self.use_atom_padding = use_atom_padding
        self.precision = precision
        self.device = torch.device(device)

        prep = deepcopy(OrderedDict(preprocessing))
        layers = []
        if cutoff is not None:
            gp = {"cutoff": cutoff, "graph_key": "graph"}
            keys = list(prep.keys())
            if keys and keys[0] == "graph":
                gp.update(prep.pop("graph"))
            gp.update(graph_config)
            layers.append(GraphGenerator(**gp))
        for name, params in prep.items():
            params = dict(params)
            key = str(params.pop("module_name")) if "module_name" in params else name
            key = str(params.pop("FID")) if "FID" in params else key
            if key.upper() not in PREPROCESSING:
                raise NotImplementedError(f"preprocessing {key!r} is outside the CUDA energy path")
            layers.append(PREPROCESSING[key.upper()](**params))

        props = {}
        for layer in layers:
            if not hasattr(layer, "get_graph_properties"):
                continue
            for k, v in layer.get_graph_properties().items():
                props[k] = {**props.get(k, {}), **v}
        self._graphs_properties = props

        self.aev_module, self.net_module = None, None
        names = []
        for name, params in deepcopy(OrderedDict(modules)).items():
            params = dict(params)
            key = str(params.pop("module_name")) if "module_name" in params else name
            key = str(params.pop("FID")) if "FID" in params else key
            if name in names:
                raise ValueError(f"Module {name} already exists")
            names.append(name)
            if key.upper() not in MODULES:
                raise NotImplementedError(f"module {key!r} is outside the CUDA energy path "
                                          f"(supported: {sorted(MODULES)})")
            cls = MODULES[key.upper()]
            fields = {f.name for f in dataclasses.fields(cls)}
            if "_graphs_properties" in fields:
                params["_graphs_properties"] = props
            params["name"] = name
            mod = cls(**params)
            if isinstance(mod, ANIAEV):
                self.aev_module = mod
            elif isinstance(mod, SpeciesIndexNet):
                self.net_module = mod
        if self.aev_module is None or self.net_module is None:
            raise NotImplementedError("the CUDA path evaluates ANI_AEV followed by SPECIES_INDEX_NET")
        net, aev = self.net_module, self.aev_module
        if net.input_key != aev.embedding_key:
            raise ValueError("SPECIES_INDEX_NET must read the ANI_AEV embedding")
        if net.output_dim != 1 or not net.use_bias or len(net.hidden()) != 3:
            raise NotImplementedError("the CUDA networks have three biased hidden layers and one output")
        if set(net.species()) != set(aev.species()):
            raise NotImplementedError("network and AEV species lists differ")
        self.aev_config = aev.config()
        self.mlp_config = MLPConfig(hidden=net.hidden(), output_dim=1, celu_alpha=net.celu_alpha())
        if self.energy_terms is not None:
            for term in self.energy_terms:
                if term != net.out_key:
                    raise NotImplementedError(f"energy term {term!r} is not produced on the CUDA path")

        self.preprocessing = PreprocessingChain(layers, use_atom_padding, self.device,
                                                self.aev_config.species_order)
        self.preproc_state = self.preprocessing.init()
        self._sized = False
        if variables is None:
            seed = 0 if rng_key is None else int(np.asarray(rng_key).reshape(-1)[-1])
            w = init_weights(self.aev_config, self.mlp_config, seed=seed)
            variables = weights_to_variables(w, net.name)[0]
        self.variables = variables
        self._pot_cache: Dict[int, Tuple[Any, ANIPotential]] = {}
        self._ws_cache = None
        # sized calls replay a CUDA graph of the whole call (False: launch
        # kernel by kernel, same results)
        self.use_cuda_graphs = True
        self._graphs: Dict[tuple, dict] = {}
        self._graph_warm: Dict[tuple, Any] = {}
        if example_data is not None:
            self.preprocess(**example_data)

    # ------------------------------------------------------------ helpers
    def weights(self, variables=None):
        """The species networks of ``variables`` (default: the model's) as
        ``[model][symbol] = [(kernel, bias), ...]`` float64 arrays."""
        variables = self.variables if variables is None else variables
        trees = variables if isinstance(variables, (list, tuple)) else [variables]
        return variables_to_weights(trees, self.aev_config.species_order, self.net_module.name)

    def _potential(self, variables) -> ANIPotential:
        key = id(variables)
        hit = self._pot_cache.get(key)
        if hit is not None and hit[0] is variables:
            return hit[1]
        weights = self.weights(variables)
        pot = ANIPotential(self.aev_config, self.mlp_config, weights=weights,
                           precision=self.precision, device=self.device)
        self._pot_cache = {key: (variables, pot)}
        self._ws_cache = None
        return pot

    def _workspace(self, pot: ANIPotential, layout: BatchLayout) -> Workspace:
        if self._ws_cache is None or self._ws_cache[0] is not layout or self._ws_cache[1] is not pot:
            # captured calls use the workspace they were captured with
            self._graphs.clear()
            self._graph_warm.clear()
            self._ws_cache = (layout, pot, Workspace(pot, layout))
        return self._ws_cache[2]

    def _stage_buffer(self, n: int, cap: int) -> Optional[torch.Tensor]:
        """Per-centre staging for the forward/adjoint pair of one call (the
        forward saves each centre's sorted neighbourhood, the adjoint reads it
        back instead of gathering and sorting again); kept across calls of the
        same size, None above 4 GB."""
        hit = getattr(self, "_stage_cache", None)
        if hit is not None and hit[0] == (n, cap):
            return hit[1]
        nbytes = int(_lib.load().fennol_aev_stage_bytes(max(n, 1), cap))
        buf = torch.empty(nbytes, dtype=torch.uint8, device=self.device) if nbytes <= (4 << 30) else None
        self._stage_cache = ((n, cap), buf)
        return buf

    def _unit_factor(self, unit) -> float:
        if unit is None:
            return 1.0
        return energy_multiplier(unit) / self.Ha_to_model_energy

    # -------------------------------------------------------------- API
    def preprocess(self, use_gpu: bool = False, verbose: bool = False, **inputs) -> Dict[str, Any]:
        """Apply the preprocessing chain.  ``use_gpu=True`` follows the
        reference's fixed-capacity path (``process`` then
        ``check_reallocate``); otherwise the host path grows capacities as it
        goes.  Both build the lists on the GPU."""
        if use_gpu and self._sized:
            inputs = self.preprocessing.check_input(inputs)
            out = self.preprocessing.process(self.preproc_state, inputs)
            state, state_up, out, overflow = self.preprocessing.check_reallocate(
                self.preproc_state, out)
            if verbose and overflow:
                print("GPU preprocessing: nblist overflow => reallocating nblist")
                print("size updates:", state_up)
        else:
            state, out = self.preprocessing(self.preproc_state, inputs)
            self._sized = True
        self.preproc_state = state
        return out

    def _prepare(self, gpu_preprocessing: bool, inputs):
        """Preprocessing for one evaluation.  Once the chain has sized its
        capacities, its layers run at those capacities (``process``) and the
        graph layers' overflow words are read together with the evaluation's
        own status, one host synchronisation per call.  Returns the processed
        inputs and the device status words still to check (None when the
        capacities were checked already)."""
        if not self._sized:
            return self.preprocess(use_gpu=gpu_preprocessing, **inputs), None
        chain = self.preprocessing
        out = chain.process(self.preproc_state, chain.check_input(inputs))
        if any(key.endswith("_overflow") and val is True for key, val in out.items()):
            return self.preprocess(use_gpu=gpu_preprocessing, **inputs), None
        return out, _status_tensors(out)

    def _status_host(self, rows: int) -> torch.Tensor:
        buf = getattr(self, "_status_pinned", None)
        if buf is None or buf.shape[0] < rows:
            buf = torch.zeros((max(rows, 4), _lib.STATUS_WORDS), dtype=torch.int32).pin_memory()
            self._status_pinned = buf
        return buf

    def _run(self, variables, gpu_preprocessing: bool, inputs, **want):
        """Preprocess and evaluate; a capacity that overflowed at the sized
        capacities reruns the call through the growing preprocessing path."""
        if variables is None:
            variables = self.variables
        if self.use_cuda_graphs and self._sized and self.device.type == "cuda":
            out = self._run_graph(variables, inputs, want)
        else:
            prepared, pending = self._prepare(gpu_preprocessing, inputs)
            out = self._evaluate(variables, prepared, pending=pending, **want)
        if out is None:
            self._graphs.clear()
            prepared = self.preprocess(use_gpu=gpu_preprocessing, **inputs)
            out = self._evaluate(variables, prepared, **want)
        return out

    def _run_graph(self, variables, inputs, want):
        """A sized call replayed from a CUDA graph: the graph layers, the
        evaluation, the output copies and the status copies, captured once per
        batch layout, capacities, weights and outputs asked for (the last few
        are kept).  Per call the host checks the inputs, copies the
        coordinates in, replays, copies the outputs out and reads the status
        words once.  Returns None when the call must take the eager path (a
        host-side overflow, or a graph capacity that overflowed)."""
        chain = self.preprocessing
        inp = chain.check_input(inputs)
        layout = inp["_layout"]
        pot = self._potential(variables)
        caps = tuple(tuple(sorted((k, v) for k, v in st.items() if isinstance(v, (int, float))))
                     for st in self.preproc_state["layers_state"])
        key = (id(layout), id(pot), caps, tuple(sorted(want.items())), self.energy_terms is None)
        entry = self._graphs.get(key)
        if entry is not None and (entry["layout"] is not layout or entry["pot"] is not pot):
            entry = None
        if entry is None and self._graph_warm.get(key) is not layout:
            # the first call of a kind runs kernel by kernel: it creates the
            # layout's cell plans and buffers that a capture must find ready
            self._graph_warm[key] = layout
            prepared = chain.process(self.preproc_state, inp)
            if any(k.endswith("_overflow") and v is True for k, v in prepared.items()):
                return None
            return self._evaluate(variables, prepared, pending=_status_tensors(prepared), **want)
        if entry is None:
            coords = inp["_coords"].clone()
            staged = {**inp, "_coords": coords}
            # everything the capture needs is created before it starts
            self._workspace(pot, layout)
            self._status_host(2 + sum(1 for layer in chain.layers if hasattr(layer, "graph_key")))
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                prepared = chain.process(self.preproc_state, staged)
                host_overflow = any(k.endswith("_overflow") and v is True for k, v in prepared.items())
                pending = _status_tensors(prepared)
                launched = self._launch(variables, prepared, pending=pending, **want)
            if host_overflow:
                return None
            entry = {"graph": g, "coords": coords, "launched": launched, "layout": layout, "pot": pot}
            while len(self._graphs) >= 4:
                self._graphs.pop(next(iter(self._graphs)))
            self._graphs[key] = entry
        else:
            entry["coords"].copy_(inp["_coords"], non_blocking=True)
        entry["graph"].replay()
        out, nwords, host, ws = entry["launched"]
        # fresh output tensors for the caller: the graph's own are rewritten by
        # the next replay
        user = dict(out)
        for k in (self.net_module.out_key, "total_energy", "forces", "virial_tensor",
                  self.aev_module.embedding_key):
            if isinstance(user.get(k), torch.Tensor):
                user[k] = user[k].clone()
        user.update({k: v for k, v in inp.items() if not k.startswith("_")})  # this call's inputs
        return self._finish(user, nwords, host, ws)

    def _evaluate(self, variables, inputs, want_forces: bool, want_embedding: bool = False,
                  want_virial: bool = False, pending=None):
        launched = self._launch(variables, inputs, want_forces, want_embedding, want_virial, pending)
        return self._finish(*launched)

    def _launch(self, variables, inputs, want_forces: bool, want_embedding: bool = False,
                want_virial: bool = False, pending=None):
        """Enqueue one evaluation: the kernels, the output copies and the copy
        of every status word to pinned host memory (nothing waits)."""
        pot = self._potential(variables)
        layout: BatchLayout = inputs["_layout"]
        ws = self._workspace(pot, layout)
        rows: NeighborRows = inputs[self.aev_module.graph_key]["rows"]
        st = _stream(self.device)
        ws.status.zero_()
        call("fennol_pack_atoms", inputs["_coords"].data_ptr(), layout.t_species.data_ptr(), layout.n,
             ws.xyzs.data_ptr(), st)
        view = _RowsView(rows)
        if want_forces and not want_virial:
            view.aev_stage = self._stage_buffer(layout.n, rows.capacity)
        pot.launch_forces(layout, view, ws, st, want_forces, want_virial)
        # the outputs are enqueued before the status read, so that one host
        # synchronisation covers them too
        out = dict(inputs)
        net_key = self.net_module.out_key
        out[net_key] = ws.e_atom.clone()
        if self.energy_terms is None:
            out["total_energy"] = torch.zeros(layout.nsys, dtype=torch.float64, device=self.device)
        else:
            out["total_energy"] = ws.energy.clone()
        if want_forces:
            f = torch.empty((layout.n, 3), dtype=torch.float32, device=self.device)
            call("fennol_forces_finalize", ws.forces4.data_ptr(), layout.n, 1.0, f.data_ptr(), st)
            out["forces"] = f if self.energy_terms is not None else torch.zeros_like(f)
        if want_virial:
            vir = ws.virial.clone()
            out["virial_tensor"] = vir if self.energy_terms is not None else torch.zeros_like(vir)
        if want_embedding:
            out[self.aev_module.embedding_key] = _embedding_from_rows(ws, layout,
                                                                       self.aev_config.aev_length)
        # every status word of the call in one read: the evaluation's, the
        # MLP kernel's error word and the graph layers' overflow words
        words = [ws.status] + list(pending or ())
        host = self._status_host(len(words) + 1)
        for k, w in enumerate(words):
            host[k].copy_(w, non_blocking=True)
        mlp_err = host[len(words), :1]
        if pot.precision != _lib.MLP_FP32:
            mlp_err.copy_(ws.mlp_ws[:4].view(torch.int32), non_blocking=True)
        else:
            mlp_err.zero_()
        return out, len(words), host, ws

    def _finish(self, out, nwords: int, host: torch.Tensor, ws: Workspace):
        """Wait for a launched evaluation and check its status words: None
        when a graph capacity overflowed (the call must rerun), the outputs
        otherwise."""
        torch.cuda.current_stream(self.device).synchronize()
        host_words = host[:nwords + 1].numpy().copy()
        status, graph_words = host_words[0], host_words[1:nwords]
        if int(host_words[nwords, 0]):
            ws.mlp_ws[:4].view(torch.int32).zero_()
            raise _lib.KernelTimeout("species MLP: a bounded wait inside the tensor-core kernel ran out")
        if graph_words.size and (graph_words[:, _lib.ST_NBR_OVERFLOW].any()
                                 or graph_words[:, _lib.ST_FILTER_OVERFLOW].any()):
            return None
        if status[_lib.ST_NONFINITE]:
            raise _lib.NonFiniteError("non-finite positions, energies or forces")
        if status[_lib.ST_ANG_OVERFLOW]:
            raise RuntimeError(f"more than {_lib.MAX_ANGULAR_NEIGHBORS} angular neighbours "
                               f"({int(status[_lib.ST_ANG_MAXCOUNT])}) around one atom")
        for k in ("_layout", "_coords"):
            out.pop(k, None)
        return out

    def __call__(self, variables=None, gpu_preprocessing: bool = False, **inputs) -> Dict[str, Any]:
        """Preprocess and apply the modules; the output holds the embedding
        (float32, [N, F] in atom order), atomic energies and total energy."""
        return self._run(variables, gpu_preprocessing, inputs, want_forces=False, want_embedding=True)

    def total_energy(self, variables=None, unit=None, gpu_preprocessing: bool = False, **inputs):
        out = self._run(variables, gpu_preprocessing, inputs, want_forces=False)
        return _scaled(out["total_energy"], self._unit_factor(unit)), out

    def energy_and_forces(self, variables=None, unit=None, gpu_preprocessing: bool = False, **inputs):
        """Total energies [B] (float64) and forces [N, 3] (float32) in the
        model's energy unit (per Angstrom), or in ``unit``."""
        out = self._run(variables, gpu_preprocessing, inputs, want_forces=True)
        fac = self._unit_factor(unit)
        return _scaled(out["total_energy"], fac), _scaled(out["forces"], fac), out

    def energy_and_forces_and_virial(self, variables=None, unit=None, gpu_preprocessing: bool = False,
                                     **inputs):
        """Energies, forces and ``virial_tensor`` [B, 3, 3] = dE/dS of the
        deformation x -> x S, cell -> cell S at S = 1 (``fennix.py:320-347``)."""
        out = self._run(variables, gpu_preprocessing, inputs, want_forces=True, want_virial=True)
        fac = self._unit_factor(unit)
        return (_scaled(out["total_energy"], fac), _scaled(out["forces"], fac),
                _scaled(out["virial_tensor"], fac), out)

    def set_energy_terms(self, energy_terms, jit: bool = True) -> None:
        """Select the energy terms of ``total_energy`` (``fennix.py:180-270``):
        a name or a list of names; None or an empty list gives zero energies
        and forces.  ``jit`` is accepted for signature compatibility."""
        if isinstance(energy_terms, str):
            energy_terms = [energy_terms]
        self.energy_terms = list(energy_terms) if energy_terms else None

    def get_model(self):
        return (self.aev_module, self.net_module), self.variables

    def get_preprocessing(self):
        return self.preprocessing, self.preproc_state

    def to_dict(self, convert_numpy: bool = False):
        return {**self._input_args, "energy_terms": self.energy_terms,
                "variables": deepcopy(self.variables)}

    def save(self, filename):
        """Write the model as ``FENNIX.save`` does (msgpack ``.fnx`` or pickle)."""
        save_model_dict(self.to_dict(), filename)

    @classmethod
    def load(cls, filename, use_atom_padding: bool = False, graph_config={}, **kwargs):
        """Read a model written by ``FENNIX.save``."""
        state = load_model_dict(filename)
        state.update(kwargs)
        return cls(**state, graph_config=graph_config, use_atom_padding=use_atom_padding)


class _RowsView:
    """The attributes :meth:`ANIPotential.launch_forces` reads of a list."""

    def __init__(self, rows: NeighborRows):
        self.rad_j, self.rad_s, self.rad_n, self.cap_r = rows.j, rows.shift, rows.count, rows.capacity
        self.aev_stage = None  # one-off rows: the plain forward/adjoint pair


def _embedding_from_rows(ws: Workspace, layout: BatchLayout, width: int) -> torch.Tensor:
    rows = layout.t_atom_row.long()
    x = ws.x[rows, :width].float()
    if ws.x_lo is not None:
        x = x + ws.x_lo[rows, :width].float()
    return x


def graph_edges(inputs: Dict[str, Any], graph_key: str = "graph") -> Dict[str, np.ndarray]:
    """The reference's edge-list view of a graph (``preprocessing.py:326-345``):
    directed ``edge_src``, ``edge_dst``, integer ``pbc_shifts`` and squared
    distances ``d12`` of every pair in the neighbour rows, as host arrays.
    Edges are listed by source atom (the reference lists i<j pairs then their
    mirror images); the set of pairs is the same."""
    rows: NeighborRows = inputs[graph_key]["rows"]
    j = rows.j.cpu().numpy()
    cnt = rows.count.cpu().numpy()
    sh = rows.shift.cpu().numpy()
    n = cnt.shape[0]
    mask = np.arange(j.shape[1])[None, :] < cnt[:, None]
    src = np.repeat(np.arange(n, dtype=np.int32), cnt)
    dst = j[mask].astype(np.int32)
    p = sh[mask].astype(np.int64) & 0xFFFFFF
    s = np.stack([(p >> (8 * k)) & 0xFF for k in range(3)], -1)
    s = np.where(s >= 128, s - 256, s).astype(np.float32)
    coords = np.asarray(_host(inputs["coordinates"]), dtype=np.float32).reshape(-1, 3)
    vec = coords[dst] - coords[src]
    if "cells" in inputs:
        cells = np.asarray(inputs["cells"], dtype=np.float32).reshape(-1, 3, 3)
        b = np.asarray(inputs["batch_index"])[src]
        cb = cells[b] if cells.shape[0] > 1 else np.broadcast_to(cells[0], (src.shape[0], 3, 3))
        vec = vec + np.einsum("ej,eji->ei", s, cb)
    return {"edge_src": src, "edge_dst": dst, "pbc_shifts": s, "d12": (vec ** 2).sum(-1)}
