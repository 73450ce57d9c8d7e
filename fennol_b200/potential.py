"""Host side of the energy/force path: batch layout, device buffers, launches.

:class:`ANIPotential` owns the packed weights of an (ensemble of) ANI-2x-style
species networks and evaluates energies and forces of batches of systems
through the C ABI.  It reproduces what FeNNol does for the same model
(``FENNIX._energy_and_forces``, ``src/fennol/models/fennix.py:260-272``): the
GRAPH / GRAPH_FILTER / GRAPH_ANGULAR_EXTENSION / SPECIES_INDEXER preprocessing
(``preprocessing.py``), ``ANIAEV`` (``embeddings/ani.py``) and
``SpeciesIndexNet`` (``misc/nets.py``), the energy sum and ``-dE/dx``.

Capacity handling follows the reference's overflow protocol
(``check_reallocate``, ``preprocessing.py:357-367``): kernels report overflow
through device status words, the host regrows with a margin
(``mult_size`` 1.05 + ``add_neigh``) and relaunches.
"""

from __future__ import annotations

import dataclasses
import math
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from ._lib import call
from .params import AEVConfig, MLPConfig, Weights, init_weights

HARTREE_TO_KCALMOL = 627.5096080305927
TILE = 128
MAX_ROW = 512            # longest neighbour row the AEV kernels stage on chip
MOLECULE_ROW_GUESS = 96  # first row length for molecules (regrown on overflow)


def _ceil(a: int, b: int) -> int:
    return (a + b - 1) // b * b


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def _stream(device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def round_weights_bf16(weights: Weights) -> Weights:
    """Round every kernel to the nearest bfloat16 (biases kept)."""
    out = []
    for model in weights:
        m = {}
        for sym, layers in model.items():
            m[sym] = [(torch.tensor(w).to(torch.bfloat16).to(torch.float64).numpy(), b)
                      for (w, b) in layers]
        out.append(m)
    return out


def pow2_scale(a: np.ndarray) -> float:
    """The power of two that brings the largest |a| into [1, 2) (1 for zeros)."""
    m = float(np.max(np.abs(a))) if a.size else 0.0
    return 1.0 if m == 0.0 else float(2.0 ** (-math.floor(math.log2(m))))


def split16(W: torch.Tensor, dtype) -> Tuple[torch.Tensor, torch.Tensor]:
    """W (float64) as hi + lo of a 16-bit type, each rounded to nearest."""
    hi = W.to(dtype)
    lo = (W - hi.to(torch.float64)).to(dtype)
    return hi, lo


class PackedMLP:
    """Device copies of the species networks in the layouts the kernels read
    (see ``fennol_mlp_weights`` in ``include/fennol_b200.h``).

    The FP16 forms store every kernel of layers 1-3 multiplied by a power of
    two per (model, species) group that puts its largest entry in [1, 2), so
    that the float16 hi + lo split keeps about 22 bits of each weight; the
    scales go to the kernel in ``f16_scale`` together with the power of two
    applied to the last layer inside the input-gradient GEMMs."""

    def __init__(self, weights: Weights, aev: AEVConfig, mlp: MLPConfig, device, precision: int):
        self.n_models = len(weights)
        self.n_species = aev.num_species
        real = [aev.aev_length, *mlp.hidden, mlp.output_dim]
        if mlp.output_dim != 1:
            raise ValueError("the energy network must have one output")
        dims = [_ceil(d, 64) for d in real[:-1]] + [1]
        self.real_dims, self.dims = real, dims
        G = self.n_models * self.n_species
        f16 = precision in _lib.F16_FORMS
        half = torch.float16 if f16 else torch.bfloat16
        scales = np.ones((G, 4))
        w32, b32, wt_hi, wt_lo, w_hi, w_lo = [], [], [], [], [], []
        for l in range(4):
            W = np.zeros((G, dims[l], dims[l + 1]))
            B = np.zeros((G, dims[l + 1]))
            for m, model in enumerate(weights):
                for s, sym in enumerate(aev.species_order):
                    k, b = model[sym][l]
                    if k.shape != (real[l], real[l + 1]):
                        raise ValueError(f"layer {l + 1} of {sym}: shape {k.shape}, expected "
                                         f"{(real[l], real[l + 1])}")
                    W[m * self.n_species + s, :real[l], :real[l + 1]] = k
                    B[m * self.n_species + s, :real[l + 1]] = b
            Wt = torch.tensor(W, dtype=torch.float64)
            w32.append(Wt.to(torch.float32).to(device).contiguous())
            b32.append(torch.tensor(B, dtype=torch.float32, device=device).contiguous())
            if f16:
                # scales of the float32 kernel the other forms evaluate
                W32 = W.astype(np.float32).astype(np.float64)
                for g in range(G):
                    scales[g, l] = pow2_scale(W32[g])
                Wt = torch.tensor(W32 * scales[:, l][:, None, None], dtype=torch.float64)
            if precision != _lib.MLP_FP32 and l < 3:
                hi, lo = split16(Wt, half)
                w_hi.append(hi.to(device).contiguous())
                w_lo.append(lo.to(device).contiguous())
                wt_hi.append(hi.transpose(1, 2).contiguous().to(device))
                wt_lo.append(lo.transpose(1, 2).contiguous().to(device))
            else:
                w_hi.append(None), w_lo.append(None), wt_hi.append(None), wt_lo.append(None)
        self.scales = (torch.tensor(scales, dtype=torch.float32, device=device).contiguous() if f16 else None)
        self._keep = (w32, b32, wt_hi, wt_lo, w_hi, w_lo)
        s = _lib.MLPWeights()
        s.n_models = self.n_models
        s.n_species = self.n_species
        for k in range(5):
            s.dims[k] = dims[k]
        s.celu_alpha = mlp.celu_alpha
        for l in range(4):
            s.w32[l] = _ptr(w32[l])
            s.b32[l] = _ptr(b32[l])
            s.wt_hi[l] = _ptr(wt_hi[l])
            s.wt_lo[l] = _ptr(wt_lo[l])
            s.w_hi[l] = _ptr(w_hi[l])
            s.w_lo[l] = _ptr(w_lo[l])
        s.f16_scale = _ptr(self.scales)
        self.struct = s


def aev_params(cfg: AEVConfig) -> _lib.AEVParams:
    p = _lib.AEVParams()
    p.num_species = cfg.num_species
    p.radial_divisions = cfg.radial_dist_divisions
    p.angular_divisions = cfg.angular_dist_divisions
    p.angle_sections = cfg.angle_sections
    p.radial_cutoff = cfg.radial_cutoff
    p.angular_cutoff = cfg.angular_cutoff
    p.radial_eta = cfg.radial_eta
    p.angular_eta = cfg.angular_eta
    p.zeta = cfg.zeta
    p.radial_start = cfg.radial_start
    p.angular_start = cfg.angular_start
    return p


def min_image_ok(cell, reach: float) -> bool:
    """Minimum image finds every pair within ``reach`` when each perpendicular
    width of the cell is at least ``2 * reach``."""
    if cell is None:
        return True
    recip = np.linalg.inv(np.asarray(cell, np.float64).reshape(3, 3))
    widths = 1.0 / np.linalg.norm(recip, axis=0)
    return bool(np.all(widths >= 2.0 * reach))


@dataclasses.dataclass
class Capacities:
    """Row lengths of the neighbour lists (reference state keys ``npairs``,
    ``npairs_skin``, ``max_neigh``)."""

    skin: int = 0
    radial: int = 0


class BatchLayout:
    """Static description of a batch: systems, cells, species-sorted rows.

    ``minimum_image`` is one flag for every periodic system or one per
    system (minimum image when true, general periodic images otherwise).
    ``reciprocal_cells`` (optional, like the reference's input key): used as
    given, cast to float32; otherwise each cell is inverted in the precision
    the caller passed it in and the inverse cast to float32, as the
    reference's ``check_input`` does (``preprocessing.py:1780-1781``)."""

    def __init__(self, species_idx: np.ndarray, natoms: Sequence[int], cells=None,
                 minimum_image: bool = True, device="cuda", reciprocal_cells=None):
        species_idx = np.asarray(species_idx, dtype=np.int32)
        natoms = np.asarray(natoms, dtype=np.int64).reshape(-1)
        n = int(natoms.sum())
        if species_idx.shape[0] != n:
            raise ValueError("species and natoms disagree")
        B = natoms.shape[0]
        self.natoms = natoms
        self.n = n
        self.nsys = B
        self.device = torch.device(device)
        start = np.concatenate([[0], np.cumsum(natoms)]).astype(np.int32)
        self.sys_start_host = start
        atom_sys = np.repeat(np.arange(B, dtype=np.int32), natoms)
        cell_arr = np.zeros((B, 3, 3), np.float32)
        recip_arr = np.zeros((B, 3, 3), np.float32)
        mode = np.zeros(B, np.int32)
        if cells is not None:
            cl = cells if isinstance(cells, (list, tuple)) else list(np.asarray(cells).reshape(-1, 3, 3))
            if len(cl) == 1 and B > 1:
                cl = cl * B
            rl = None
            if reciprocal_cells is not None:
                rl = list(np.asarray(reciprocal_cells).reshape(-1, 3, 3))
                if len(rl) == 1 and B > 1:
                    rl = rl * B
            for b, c in enumerate(cl):
                if c is None:
                    continue
                c = np.asarray(c).reshape(3, 3)
                cell_arr[b] = c.astype(np.float32)
                recip_arr[b] = (np.linalg.inv(c) if rl is None else rl[b]).astype(np.float32)
                mi = minimum_image[b] if isinstance(minimum_image, (list, tuple, np.ndarray)) \
                    else minimum_image
                mode[b] = _lib.PBC_MINIMUM_IMAGE if mi else _lib.PBC_GENERAL
        self.has_pbc = bool((mode != 0).any())
        # species present in the batch (bit s): the AEV columns of absent
        # species and species pairs are zero in every row
        self.species_mask = int(np.bitwise_or.reduce(1 << np.unique(np.asarray(species_idx, np.int64)))) \
            if n else 1
        self.mode_host, self.cell_host, self.recip_host = mode, cell_arr, recip_arr
        # species-sorted rows, segments padded to the 128-row tile
        self.species_idx = species_idx
        S = int(species_idx.max()) + 1 if n else 1
        row = np.zeros(n, np.int32)
        tiles_s, tiles_r = [], []
        self.species_segments: List[Tuple[int, int, int]] = []  # (species, first row, atoms)
        off = 0
        for s in range(max(S, 1)):
            idx = np.nonzero(species_idx == s)[0]
            if idx.size == 0:
                continue
            row[idx] = off + np.arange(idx.size)
            self.species_segments.append((s, off, int(idx.size)))
            for t in range((idx.size + TILE - 1) // TILE):
                tiles_s.append(s)
                tiles_r.append(off + t * TILE)
            off += _ceil(idx.size, TILE)
        self.rows = max(off, TILE)
        self.ntiles = len(tiles_s)
        self.atom_row_host = row
        dev = self.device
        self.t_atom_sys = torch.tensor(atom_sys, device=dev)
        self.t_sys_start = torch.tensor(start, device=dev)
        self.t_mode = torch.tensor(mode, device=dev)
        self.t_cell = torch.tensor(cell_arr.reshape(B, 9), device=dev)
        self.t_recip = torch.tensor(recip_arr.reshape(B, 9), device=dev)
        self.t_species = torch.tensor(species_idx, device=dev)
        self.t_atom_row = torch.tensor(row, device=dev)
        self.t_tile_species = torch.tensor(np.asarray(tiles_s, np.int32), device=dev)
        self.t_tile_row = torch.tensor(np.asarray(tiles_r, np.int32), device=dev)
        self._plans: Dict[float, Tuple[torch.Tensor, torch.Tensor, int]] = {}

    def plan(self, cutoff: float):
        """Cell grid for a cutoff (``fennol_graph_plan``), cached."""
        key = float(cutoff)
        if key not in self._plans:
            import ctypes as C
            grid = np.zeros((self.nsys, 4), np.int32)
            nrep = np.zeros((self.nsys, 3), np.int32)
            total = call("fennol_graph_plan", self.nsys, self.mode_host.ctypes.data,
                         self.recip_host.ctypes.data, key, grid.ctypes.data, nrep.ctypes.data)
            self._plans[key] = (torch.tensor(grid, device=self.device),
                                torch.tensor(nrep, device=self.device), int(total))
        return self._plans[key]

    def estimate_capacity(self, cutoff: float) -> int:
        """Initial row length: the largest system size for molecules, the
        density estimate with a 25% margin for periodic boxes."""
        best = 8
        for b in range(self.nsys):
            nb = int(self.natoms[b])
            if self.mode_host[b] == 0:
                # molecules: bounded by the size, and by a dense-liquid count
                # (overflow regrows the rows)
                best = max(best, min(nb - 1, MOLECULE_ROW_GUESS))
            else:
                vol = abs(float(np.linalg.det(self.cell_host[b].astype(np.float64))))
                est = 4.0 / 3.0 * math.pi * cutoff ** 3 * nb / max(vol, 1e-9)
                best = max(best, int(est * 1.25) + 16)
        return min(_ceil(max(best, 8), 8), MAX_ROW)


class GraphBuffers:
    """Neighbour rows of one layout: the build list (cutoff + skin) and, when
    a skin is used, the radial list filtered from it.  With ``stage`` also the
    per-centre AEV staging that the forward saves for the adjoint of the same
    call (``fennol_aev_forward_staged``): worth its memory for buffers reused
    over many calls (MD, a repeated single-point layout), not for one-off
    batches."""

    def __init__(self, layout: BatchLayout, cutoff: float, skin: float, cap: int, cap_radial: int,
                 stage: bool = False):
        dev = layout.device
        n = max(layout.n, 1)
        self.cutoff, self.skin = cutoff, skin
        self.cap = cap
        self.nbr_j = torch.zeros((n, cap), dtype=torch.int32, device=dev)
        self.nbr_s = torch.zeros((n, cap), dtype=torch.int32, device=dev)
        self.nbr_n = torch.zeros(n, dtype=torch.int32, device=dev)
        grid, nrep, ncells = layout.plan(cutoff + skin)
        self.grid, self.nrep, self.ncells = grid, nrep, ncells
        ws = _lib.load().fennol_graph_workspace_bytes(n, ncells)
        self.ws = torch.zeros(int(ws), dtype=torch.uint8, device=dev)
        if skin > 0:
            self.cap_r = cap_radial
            self.rad_j = torch.zeros((n, cap_radial), dtype=torch.int32, device=dev)
            self.rad_s = torch.zeros((n, cap_radial), dtype=torch.int32, device=dev)
            self.rad_n = torch.zeros(n, dtype=torch.int32, device=dev)
        else:
            self.cap_r = cap
            self.rad_j, self.rad_s, self.rad_n = self.nbr_j, self.nbr_s, self.nbr_n
        self.aev_stage = None
        if stage:
            sb = _lib.load().fennol_aev_stage_bytes(n, self.cap_r)
            self.aev_stage = torch.empty(int(sb), dtype=torch.uint8, device=dev)

    def regrown(self, layout: BatchLayout, cap: int, cap_radial: int) -> "GraphBuffers":
        """New buffers with larger row capacities and the same settings."""
        return GraphBuffers(layout, self.cutoff, self.skin, cap, cap_radial, stage=self.aev_stage is not None)

    def build(self, layout: BatchLayout, coords: torch.Tensor, status: torch.Tensor, stream: int,
              enable_flag: Optional[torch.Tensor] = None):
        call("fennol_graph_build", coords.data_ptr(), layout.n, layout.t_atom_sys.data_ptr(), layout.nsys,
             layout.t_sys_start.data_ptr(), layout.t_mode.data_ptr(), layout.t_cell.data_ptr(),
             layout.t_recip.data_ptr(), self.grid.data_ptr(), self.nrep.data_ptr(), self.ncells,
             float(self.cutoff + self.skin), self.cap, self.nbr_j.data_ptr(), self.nbr_s.data_ptr(),
             self.nbr_n.data_ptr(), status.data_ptr(), self.ws.data_ptr(), self.ws.numel(),
             _ptr(enable_flag), stream)

    def filter(self, layout: BatchLayout, coords: torch.Tensor, status: torch.Tensor, stream: int):
        if self.skin <= 0:
            return
        call("fennol_graph_filter", coords.data_ptr(), layout.n, layout.t_atom_sys.data_ptr(),
             layout.t_cell.data_ptr(), self.nbr_j.data_ptr(), self.nbr_s.data_ptr(), self.nbr_n.data_ptr(),
             self.cap, float(self.cutoff), self.cap_r, self.rad_j.data_ptr(), self.rad_s.data_ptr(),
             self.rad_n.data_ptr(), status.data_ptr(), stream)


class Workspace:
    """Per-layout device buffers of one energy/force evaluation."""

    def __init__(self, pot: "ANIPotential", layout: BatchLayout):
        dev = layout.device
        n = max(layout.n, 1)
        rows = layout.rows
        d0 = pot.mlp.dims[0]
        self.xyzs = torch.zeros((n, 4), dtype=torch.float32, device=dev)
        if pot.precision == _lib.MLP_FP32:
            self.x = torch.zeros((rows, d0), dtype=torch.float32, device=dev)
            self.x_lo = None
            self.aev_kind = _lib.AEV_F32
        elif pot.precision in _lib.F16_FORMS:
            self.x = torch.zeros((rows, d0), dtype=torch.float16, device=dev)
            self.x_lo = torch.zeros((rows, d0), dtype=torch.float16, device=dev)
            self.aev_kind = _lib.AEV_F16X2
        else:
            self.x = torch.zeros((rows, d0), dtype=torch.bfloat16, device=dev)
            self.x_lo = (torch.zeros((rows, d0), dtype=torch.bfloat16, device=dev)
                         if pot.precision != _lib.MLP_BF16 else None)
            self.aev_kind = _lib.AEV_BF16 if pot.precision == _lib.MLP_BF16 else _lib.AEV_BF16X2
        self.dx = torch.zeros((rows, d0), dtype=torch.float32, device=dev)
        self.e_rows = torch.zeros(rows, dtype=torch.float32, device=dev)
        mws = _lib.load().fennol_mlp_workspace_bytes(pot.precision, rows, pot.mlp.n_models,
                                                     pot.mlp.struct)
        self.mlp_ws = torch.zeros(max(int(mws), 256), dtype=torch.uint8, device=dev)
        self.forces4 = torch.zeros((n, 4), dtype=torch.float32, device=dev)
        self.forces = torch.zeros((n, 3), dtype=torch.float32, device=dev)
        self.energy = torch.zeros(layout.nsys, dtype=torch.float64, device=dev)
        self.e_atom = torch.zeros(n, dtype=torch.float64, device=dev)
        ews = _lib.load().fennol_energy_workspace_bytes(layout.n, layout.nsys)
        self.energy_ws = torch.zeros(int(ews), dtype=torch.uint8, device=dev)
        self.status = torch.zeros(_lib.STATUS_WORDS, dtype=torch.int32, device=dev)
        self.atom_virial = None
        self.virial = None

    def virial_buffers(self, layout: "BatchLayout"):
        """Per-centre (float32 [N, 9]) and per-system (float64 [B, 3, 3]) virials."""
        if self.atom_virial is None:
            dev = layout.device
            self.atom_virial = torch.zeros((max(layout.n, 1), 9), dtype=torch.float32, device=dev)
            self.virial = torch.zeros((layout.nsys, 3, 3), dtype=torch.float64, device=dev)
        return self.atom_virial, self.virial


class ANIPotential:
    """ANI-2x-style potential evaluated by the sm_100a kernels.

    ``precision``: ``"fp32"`` (CUDA-core GEMMs), ``"bf16"``, ``"bf16x2"`` or
    ``"bf16x3"`` (tcgen05 tensor-core GEMMs with 1, 2 or 3 BF16 products), or
    ``"f16x3x1"`` / ``"f16x3x2"`` (tcgen05 FP16 hi + lo splits of activations
    and scaled float32 weights: 3 products in the forward GEMMs, 1 or 2 in the
    input-gradient GEMMs; within the energy and force budgets against the
    FP64 model for float32 weights).
    ``bf16_weights`` rounds the kernels to BFloat16 (a model stored in BF16);
    bf16x2 is exact in the weights for such a model.
    ``minimum_image``: True / False force the minimum-image or the general
    periodic search; None (default) picks per system (see :meth:`layout`).
    ``use_graphs``: from the second call on the same batch (species, sizes,
    cells) the whole evaluation is one CUDA-graph launch.
    Energies are returned in Hartree (FeNNol's default model unit) and
    forces in Hartree/Angstrom, unless ``energy_unit="kcalpermol"``.
    """

    def __init__(self, aev: AEVConfig = AEVConfig(), mlp: MLPConfig = MLPConfig(),
                 weights: Optional[Weights] = None, precision: str = "fp32", device="cuda",
                 seed: int = 0, n_models: int = 1, energy_unit: str = "Ha",
                 minimum_image: Optional[bool] = None, output_scale: float = 1.0,
                 bf16_weights: bool = False, use_graphs: bool = True):
        if precision not in _lib.PRECISIONS:
            raise ValueError(f"precision must be one of {list(_lib.PRECISIONS)}")
        _lib.load()
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("ANIPotential runs on CUDA devices only")
        self.aev_cfg, self.mlp_cfg = aev, mlp
        if weights is None:
            weights = init_weights(aev, mlp, seed=seed, n_models=n_models, output_scale=output_scale)
        if bf16_weights:
            weights = round_weights_bf16(weights)
        self.weights = weights
        self.precision = _lib.PRECISIONS[precision]
        self.precision_name = precision
        self.mlp = PackedMLP(weights, aev, mlp, self.device, self.precision)
        self.params = aev_params(aev)
        if _lib.load().fennol_aev_length(C_ptr(self.params)) != aev.aev_length:
            raise ValueError("unsupported AEV hyper-parameters for the CUDA kernels")
        self.unit_scale = {"ha": 1.0, "hartree": 1.0,
                           "kcalpermol": HARTREE_TO_KCALMOL}[energy_unit.lower()]
        self.minimum_image = minimum_image
        self._cache: Dict[tuple, tuple] = {}
        self._chunk_masks: Dict[int, int] = {}
        self.capacity_margin = 1.05
        self.add_neigh = 8
        # repeated calls on the same batch replay one captured CUDA graph
        self.use_graphs = use_graphs
        self._graphs: Dict[tuple, dict] = {}
        self._calls: Dict[tuple, int] = {}

    # ------------------------------------------------------------------ layout
    def layout(self, species, natoms, cells=None, reach: Optional[float] = None) -> BatchLayout:
        """Batch layout.  With ``minimum_image=None`` each periodic system uses
        the minimum-image search when its cell is at least twice ``reach``
        (default: the radial cutoff) wide in every direction, and the general
        periodic search over cell images otherwise."""
        sidx = self.aev_cfg.species_index(np.asarray(species))
        mi = self.minimum_image
        if mi is None:
            r = self.aev_cfg.radial_cutoff if reach is None else reach
            nsys = len(np.asarray(natoms).reshape(-1))
            if cells is None:
                mi = True
            else:
                cl = cells if isinstance(cells, (list, tuple)) else list(np.asarray(cells).reshape(-1, 3, 3))
                if len(cl) == 1 and nsys > 1:
                    cl = cl * nsys
                mi = [min_image_ok(c, r) for c in cl]
        return BatchLayout(sidx, natoms, cells, mi, self.device)

    def buffers(self, layout: BatchLayout, skin: float = 0.0, cap: Optional[int] = None,
                cap_radial: Optional[int] = None):
        rc = self.aev_cfg.radial_cutoff
        if cap is None:
            cap = layout.estimate_capacity(rc + skin)
        if cap_radial is None:
            cap_radial = layout.estimate_capacity(rc) if skin > 0 else cap
        g = GraphBuffers(layout, rc, skin, cap, cap_radial, stage=True)
        ws = Workspace(self, layout)
        return g, ws

    def active_chunks(self, species_mask: int) -> int:
        """The 64-column chunks of the AEV rows that can be non-zero for a
        batch of these species (``fennol_aev_active_chunks``)."""
        m = self._chunk_masks.get(species_mask)
        if m is None:
            m = int(_lib.load().fennol_aev_active_chunks(C_ptr(self.params), species_mask))
            if m == 0:
                m = (1 << 64) - 1   # widths the mask cannot describe: every column
            self._chunk_masks[species_mask] = m
        return m

    def mlp_launches(self) -> int:
        """Kernels launched by one fennol_mlp_energy_grad call: the FP32 form
        runs 7 per model, the fused tcgen05 kernel (BF16 / BF16x2 on these
        layer sizes) one, the unfused tcgen05 path 6 per model and one sum."""
        import os
        if self.precision == _lib.MLP_FP32:
            return 7 * self.mlp.n_models
        if self.precision in _lib.F16_FORMS:
            return 1
        fused = (self.precision in (_lib.MLP_BF16, _lib.MLP_BF16X2) and self.mlp.dims[0] % 256 == 0
                 and max(self.mlp.dims[1:4]) <= 256 and not os.environ.get("FENNOL_MLP_UNFUSED"))
        return 1 if fused else 6 * self.mlp.n_models + 1

    # --------------------------------------------------------------- launches
    def launch_forces(self, layout: BatchLayout, g: GraphBuffers, ws: Workspace, stream: int,
                      want_forces: bool = True, want_virial: bool = False,
                      ghost_rows: Optional[torch.Tensor] = None, check_finite: bool = True):
        """AEV -> MLP -> energies (and adjoint -> forces) from the current radial
        list.  ``ghost_rows``: MLP rows of centres whose energy does not count
        (their row energy and dE/dAEV are cleared before the sum and the adjoint).
        ``check_finite``: one more launch sets status[ST_NONFINITE] when the
        positions, energies or forces hold a NaN or an infinity (an atom at a
        NaN position drops out of every list, so the energy alone can stay
        finite)."""
        lib_p = C_ptr(self.params)
        n = layout.n
        # the adjoint reuses the forward's staging when the buffers carry it
        staged = want_forces and not want_virial and getattr(g, "aev_stage", None) is not None
        if staged:
            call("fennol_aev_forward_staged", ws.xyzs.data_ptr(), n, layout.t_atom_sys.data_ptr(),
                 layout.t_cell.data_ptr(), g.rad_j.data_ptr(), g.rad_s.data_ptr(), g.rad_n.data_ptr(),
                 g.cap_r, lib_p, layout.t_atom_row.data_ptr(), ws.aev_kind, ws.x.data_ptr(),
                 _ptr(ws.x_lo), ws.x.shape[1], g.aev_stage.data_ptr(), g.aev_stage.numel(),
                 ws.status.data_ptr(), stream)
        else:
            call("fennol_aev_forward", ws.xyzs.data_ptr(), n, layout.t_atom_sys.data_ptr(),
                 layout.t_cell.data_ptr(), g.rad_j.data_ptr(), g.rad_s.data_ptr(), g.rad_n.data_ptr(),
                 g.cap_r, lib_p, layout.t_atom_row.data_ptr(), ws.aev_kind, ws.x.data_ptr(),
                 _ptr(ws.x_lo), ws.x.shape[1], ws.status.data_ptr(), stream)
        call("fennol_mlp_energy_grad_active", self.precision, layout.rows, layout.ntiles,
             layout.t_tile_species.data_ptr(), layout.t_tile_row.data_ptr(), C_ptr(self.mlp.struct),
             ws.x.data_ptr(), _ptr(ws.x_lo), self.active_chunks(layout.species_mask), ws.e_rows.data_ptr(),
             ws.dx.data_ptr(), ws.mlp_ws.data_ptr(), ws.mlp_ws.numel(), stream)
        if ghost_rows is not None and ghost_rows.numel() > 0:
            ws.e_rows.index_fill_(0, ghost_rows, 0.0)
            ws.dx.index_fill_(0, ghost_rows, 0.0)
        call("fennol_energy_reduce", ws.e_rows.data_ptr(), layout.t_atom_row.data_ptr(), n,
             layout.t_sys_start.data_ptr(), layout.nsys, float(self.unit_scale), ws.energy.data_ptr(),
             ws.e_atom.data_ptr(), ws.energy_ws.data_ptr(), ws.energy_ws.numel(), stream)
        if want_forces and want_virial:
            ws.forces4.zero_()
            av, vir = ws.virial_buffers(layout)
            call("fennol_aev_backward_virial", ws.xyzs.data_ptr(), n, layout.t_atom_sys.data_ptr(),
                 layout.t_cell.data_ptr(), g.rad_j.data_ptr(), g.rad_s.data_ptr(), g.rad_n.data_ptr(),
                 g.cap_r, lib_p, layout.t_atom_row.data_ptr(), ws.dx.data_ptr(), ws.dx.shape[1],
                 ws.forces4.data_ptr(), av.data_ptr(), ws.status.data_ptr(), stream)
            call("fennol_virial_reduce", av.data_ptr(), n, layout.t_sys_start.data_ptr(), layout.nsys,
                 float(self.unit_scale), vir.data_ptr(), stream)
        elif staged:
            ws.forces4.zero_()
            call("fennol_aev_backward_staged", ws.xyzs.data_ptr(), n, layout.t_atom_sys.data_ptr(),
                 layout.t_cell.data_ptr(), g.rad_j.data_ptr(), g.rad_s.data_ptr(), g.rad_n.data_ptr(),
                 g.cap_r, lib_p, layout.t_atom_row.data_ptr(), ws.dx.data_ptr(), ws.dx.shape[1],
                 ws.forces4.data_ptr(), g.aev_stage.data_ptr(), ws.status.data_ptr(), stream)
        elif want_forces:
            ws.forces4.zero_()
            call("fennol_aev_backward", ws.xyzs.data_ptr(), n, layout.t_atom_sys.data_ptr(),
                 layout.t_cell.data_ptr(), g.rad_j.data_ptr(), g.rad_s.data_ptr(), g.rad_n.data_ptr(),
                 g.cap_r, lib_p, layout.t_atom_row.data_ptr(), ws.dx.data_ptr(), ws.dx.shape[1],
                 ws.forces4.data_ptr(), ws.status.data_ptr(), stream)
        if check_finite:
            _lib.check_finite([ws.xyzs[:n], ws.energy, ws.forces4[:n] if want_forces else None], ws.status,
                              stream)

    def check_status(self, ws: Workspace, g: GraphBuffers) -> Optional[Tuple[int, int]]:
        """None if every list fitted, else the capacities to regrow to.
        Raises :class:`NonFiniteError` on a NaN or infinity found by the
        device check and :class:`KernelTimeout` when a bounded wait of the
        tensor-core MLP ran out (its error word is cleared first, so the next
        call starts clean)."""
        st = ws.status.cpu().numpy()
        if self.precision != _lib.MLP_FP32:
            err = ws.mlp_ws[:4].view(torch.int32)
            if int(err[0]):
                err.zero_()
                raise _lib.KernelTimeout("species MLP: a bounded wait inside the tensor-core kernel ran out "
                                         "(the launch was abandoned; its outputs are invalid)")
        if st[_lib.ST_NONFINITE]:
            raise _lib.NonFiniteError("non-finite positions, energies or forces")
        if st[_lib.ST_ANG_OVERFLOW]:
            raise RuntimeError(f"more than {_lib.MAX_ANGULAR_NEIGHBORS} angular neighbours "
                               f"({int(st[_lib.ST_ANG_MAXCOUNT])}) around one atom")
        grow = None
        if st[_lib.ST_NBR_OVERFLOW] or st[_lib.ST_FILTER_OVERFLOW]:
            cap = g.cap
            capr = g.cap_r
            if st[_lib.ST_NBR_OVERFLOW]:
                cap = int(self.capacity_margin * st[_lib.ST_NBR_MAXCOUNT]) + self.add_neigh
            if st[_lib.ST_FILTER_OVERFLOW]:
                capr = int(self.capacity_margin * st[_lib.ST_FILTER_MAXCOUNT]) + self.add_neigh
            if g.skin <= 0:
                capr = cap
            if max(cap, capr) > MAX_ROW:
                raise RuntimeError(f"neighbour rows longer than {MAX_ROW} are not supported")
            grow = (_ceil(cap, 8), _ceil(capr, 8))
        return grow

    def _get(self, key, layout_fn):
        if key not in self._cache:
            layout = layout_fn()
            g, ws = self.buffers(layout)
            self._cache = {key: (layout, g, ws)}  # one cached layout
            self._graphs, self._calls = {}, {}
        return self._cache[key]

    def energy_and_forces(self, coordinates, species, natoms=None, cells=None,
                          want_forces: bool = True, centres: Optional[int] = None):
        """Energies [B] (float64) and forces [N,3] (float32) as torch tensors
        on the device.  ``coordinates`` may be a host array or a device
        tensor ([N,3], Angstrom); ``species`` are atomic numbers.

        ``centres`` (one system only): only the first ``centres`` atoms are
        centres whose atomic energies count; the others are ghost atoms that
        only shape those centres' environments (spatial decomposition).  The
        forces are then -d/dx of the owned centres' energy, on all atoms."""
        ws = self._evaluate(coordinates, species, natoms, cells, want_forces, False, centres)
        n = self._cache[next(iter(self._cache))][0].n
        return ws.energy, (ws.forces[:n] if want_forces else None)

    def energy_forces_virial(self, coordinates, species, natoms=None, cells=None):
        """Energies [B], forces [N,3] and the virial tensor [B,3,3] (float64):
        dE/dS of the deformation x -> x S, cell -> cell S at S = 1, FeNNol's
        ``virial_tensor`` (``fennix.py:320-347``), in the energy unit."""
        ws = self._evaluate(coordinates, species, natoms, cells, True, True)
        n = self._cache[next(iter(self._cache))][0].n
        return ws.energy, ws.forces[:n], ws.virial

    def _evaluate(self, coordinates, species, natoms, cells, want_forces: bool, want_virial: bool,
                  centres: Optional[int] = None):
        species = np.asarray(species)
        if natoms is None:
            natoms = [species.shape[0]]
        natoms = tuple(int(v) for v in np.asarray(natoms).reshape(-1))
        if not (isinstance(coordinates, torch.Tensor) and coordinates.is_cuda):
            # host input: checked before upload (device inputs by the device check)
            if not np.all(np.isfinite(np.asarray(coordinates, dtype=np.float64))):
                raise ValueError("coordinates hold a NaN or an infinity")
        if centres is not None:
            if len(natoms) != 1 or not 0 <= int(centres) <= natoms[0]:
                raise ValueError("centres applies to a single system and must lie in [0, natoms]")
            centres = None if int(centres) == natoms[0] else int(centres)
        if cells is None:
            cell_key = None
        elif isinstance(cells, (list, tuple)):
            cell_key = tuple(None if c is None else np.asarray(c, np.float32).tobytes() for c in cells)
        else:
            cell_key = np.asarray(cells, dtype=np.float32).tobytes()
        key = (species.tobytes(), natoms, cell_key)
        layout, g, ws = self._get(key, lambda: self.layout(species, natoms, cells))
        coords = torch.as_tensor(coordinates, dtype=torch.float32)
        if coords.device != self.device:
            coords = coords.to(self.device, non_blocking=True)
        coords = coords.contiguous()
        stream = _stream(self.device)
        gkey = (key, bool(want_forces), bool(want_virial), centres)
        rec = self._graphs.get(gkey) if self.use_graphs else None
        if rec is not None and rec["g"] is g:
            # same batch as the last calls: one graph launch for the whole evaluation
            rec["coords"].copy_(coords, non_blocking=True)
            rec["graph"].replay()
            grow = self.check_status(ws, g)
            if grow is None:
                return ws
            self._graphs.pop(gkey, None)
            g = g.regrown(layout, grow[0], grow[1])
            self._cache[key] = (layout, g, ws)
        for _attempt in range(4):
            self._launch_all(layout, g, ws, coords, stream, want_forces, want_virial, centres)
            grow = self.check_status(ws, g)
            if grow is None:
                break
            g = g.regrown(layout, grow[0], grow[1])
            self._cache[key] = (layout, g, ws)
        else:
            raise RuntimeError("neighbour capacity did not converge")
        if self.use_graphs:
            calls = self._calls.get(gkey, 0) + 1
            self._calls = {gkey: calls}
            if calls >= 2:  # a repeated batch: capture it once
                self._capture(gkey, layout, g, ws, coords, want_forces, want_virial, centres)
        return ws

    def _launch_all(self, layout: BatchLayout, g: GraphBuffers, ws: Workspace, coords: torch.Tensor,
                    stream: int, want_forces: bool, want_virial: bool = False, centres: Optional[int] = None):
        """Every launch of one evaluation: pack, list build and filter, AEV,
        MLP, energy sum, adjoint and force finalisation."""
        ws.status.zero_()
        call("fennol_pack_atoms", coords.data_ptr(), layout.t_species.data_ptr(), layout.n,
             ws.xyzs.data_ptr(), stream)
        g.build(layout, coords, ws.status, stream)
        g.filter(layout, coords, ws.status, stream)
        ghost_rows = None if centres is None else layout.t_atom_row[centres:layout.n].long()
        self.launch_forces(layout, g, ws, stream, want_forces, want_virial, ghost_rows)
        if want_forces:
            call("fennol_forces_finalize", ws.forces4.data_ptr(), layout.n, float(self.unit_scale),
                 ws.forces.data_ptr(), stream)

    def _capture(self, gkey, layout, g, ws, coords, want_forces, want_virial, centres=None):
        buf = torch.empty_like(coords)
        buf.copy_(coords)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            self._launch_all(layout, g, ws, buf, _stream(self.device), want_forces, want_virial, centres)
        self._graphs = {gkey: {"graph": graph, "coords": buf, "g": g}}
        # the replay recomputes the same values; results of this call stay valid

    def neighbor_lists(self, coordinates, species, natoms=None, cells=None, cutoff=None):
        """Per-atom rows (j, shift, count) of the pair list for ``cutoff``
        (default: the radial cutoff) as host arrays, regrowing on overflow."""
        species = np.asarray(species)
        if natoms is None:
            natoms = [species.shape[0]]
        rc = self.aev_cfg.radial_cutoff if cutoff is None else cutoff
        layout = self.layout(species, natoms, cells, reach=rc)
        cap = layout.estimate_capacity(rc)
        coords = torch.as_tensor(np.asarray(coordinates), dtype=torch.float32).to(self.device).contiguous()
        status = torch.zeros(_lib.STATUS_WORDS, dtype=torch.int32, device=self.device)
        stream = _stream(self.device)
        for _ in range(4):
            g = GraphBuffers(layout, rc, 0.0, cap, cap)
            status.zero_()
            g.build(layout, coords, status, stream)
            st = status.cpu().numpy()
            if not st[_lib.ST_NBR_OVERFLOW]:
                return g.nbr_j.cpu().numpy(), g.nbr_s.cpu().numpy(), g.nbr_n.cpu().numpy(), layout
            cap = _ceil(int(1.05 * st[_lib.ST_NBR_MAXCOUNT]) + 8, 8)
        raise RuntimeError("neighbour capacity did not converge")


def C_ptr(struct):
    import ctypes
    return ctypes.pointer(struct)


def unpack_shifts(packed: np.ndarray) -> np.ndarray:
    """Packed signed-byte shifts (x | y<<8 | z<<16) -> int [..., 3]."""
    p = np.asarray(packed).astype(np.int64) & 0xFFFFFF
    out = np.stack([(p >> (8 * k)) & 0xFF for k in range(3)], -1)
    return np.where(out >= 128, out - 256, out)
