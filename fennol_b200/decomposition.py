"""Spatial decomposition of one large periodic box over several GPUs.

FeNNol evaluates a system on one device (``md/dynamic.py:116``); a box too
large for one GPU is cut here into P slabs along x, one per rank:

* rank r owns the atoms whose wrapped x lies in [r w, (r + 1) w), w = L_x / P;
* it also holds ghost copies of the atoms within ``halo`` (at least the
  radial cutoff, plus the skin for MD lists) of its slab's two faces, shifted
  across the periodic boundary where needed, in a local cell that is the
  slab plus both halos plus one more halo of empty space along x (so no
  periodic image along x comes within the cutoff) and the box itself along
  y and z;
* it evaluates the potential for owned + ghost atoms with only the owned
  atoms as centres (``ANIPotential.energy_and_forces(..., centres=n_owned)``
  clears the ghost centres' energies and dE/dAEV before the sum and the
  adjoint), so its energy is the sum of its owned atomic energies and its
  forces are -d/dx of that sum on owned and ghost atoms;
* the one exchange step sums every rank's forces into the global array
  (forces that landed on a ghost go to its owner) and the energies, one
  all-reduce each over ``torch.distributed`` (NCCL on GPUs, gloo on CPUs).

Positions stay replicated on every rank (N x 3 floats: 24 MB for 10^6
atoms); the neighbour lists, AEVs, MLP and adjoint, which carry the memory
and the time, are split.  An MD driver integrates the replicated positions
with the summed forces on every rank (same seed, same noise), so the ranks
stay identical without another exchange.  The slab width must be at least
the halo, and the cell orthorhombic.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Optional, Tuple

import numpy as np
import torch


@dataclass
class LocalSystem:
    ids: np.ndarray        # global atom index of each local atom: owned first, then ghosts
    coordinates: np.ndarray  # [m, 3] float64, in the local cell
    n_owned: int
    cell: np.ndarray       # [3, 3] local cell (rows are lattice vectors)


class SlabPlan:
    """Cut an orthorhombic box into ``n_ranks`` slabs along x."""

    def __init__(self, cell, n_ranks: int, halo: float):
        cell = np.asarray(cell, dtype=np.float64).reshape(3, 3)
        if np.abs(cell - np.diag(np.diag(cell))).max() > 0:
            raise ValueError("slab decomposition needs an orthorhombic cell")
        if n_ranks < 1:
            raise ValueError("n_ranks must be >= 1")
        self.cell = cell
        self.lengths = np.diag(cell).copy()
        self.n_ranks = int(n_ranks)
        self.halo = float(halo)
        self.width = self.lengths[0] / self.n_ranks
        if self.n_ranks > 1 and self.width < self.halo:
            raise ValueError(f"slab width {self.width:.3f} A is below the halo {self.halo:.3f} A: "
                             "use fewer ranks")

    def owners(self, coordinates) -> np.ndarray:
        """Owning rank of every atom."""
        xw = np.mod(np.asarray(coordinates, dtype=np.float64)[:, 0], self.lengths[0])
        return np.minimum((xw / self.width).astype(np.int64), self.n_ranks - 1)

    def local(self, coordinates, rank: int) -> LocalSystem:
        """The atoms rank ``rank`` evaluates and where they sit in its cell."""
        x = np.asarray(coordinates, dtype=np.float64)
        n = x.shape[0]
        if self.n_ranks == 1:
            return LocalSystem(np.arange(n), x.copy(), n, self.cell.copy())
        lx, w, h = self.lengths[0], self.width, self.halo
        # position along x measured from the slab's lower face, in [0, L_x)
        u = np.mod(np.mod(x[:, 0], lx) - rank * w, lx)
        owned = np.nonzero(self.owners(x) == rank)[0]
        above = np.nonzero((u >= w) & (u < w + h))[0]          # beyond the upper face
        below = np.nonzero(u >= lx - h)[0]                     # beyond the lower face (shifted by -L_x)
        ids = np.concatenate([owned, above, below])
        ux = np.concatenate([u[owned], u[above], u[below] - lx]) + h
        yz = np.mod(x[ids, 1:], self.lengths[1:])
        local_x = np.concatenate([ux[:, None], yz], axis=1)
        cell = np.diag([w + 3.0 * h, self.lengths[1], self.lengths[2]])
        return LocalSystem(ids, local_x, owned.size, cell)


def rank_contribution(pot, plan: SlabPlan, rank: int, coordinates, species) -> Tuple[torch.Tensor, torch.Tensor]:
    """Energy of the owned atoms of ``rank`` (float64 scalar) and its forces
    on all atoms (float64 [N, 3], zero away from its owned and ghost atoms),
    both on the potential's device.  Summed over the ranks they are the energy
    and forces of the whole box."""
    loc = plan.local(coordinates, rank)
    sp = np.asarray(species)[loc.ids]
    e, f = pot.energy_and_forces(loc.coordinates, sp, [loc.ids.size], loc.cell[None], centres=loc.n_owned)
    n = np.asarray(coordinates).shape[0]
    forces = torch.zeros((n, 3), dtype=torch.float64, device=f.device)
    forces.index_add_(0, torch.as_tensor(loc.ids, device=f.device), f.to(torch.float64))
    return e.to(torch.float64).sum(), forces


class SlabEnergyForces:
    """Energy and forces of one periodic box evaluated by all ranks of a
    process group, each on its slab; every rank receives the totals."""

    def __init__(self, pot, cell, halo: Optional[float] = None, group=None):
        import torch.distributed as dist

        self.pot, self.group = pot, group
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.plan = SlabPlan(cell, self.world, pot.aev_cfg.radial_cutoff if halo is None else halo)

    def __call__(self, coordinates, species) -> Tuple[torch.Tensor, torch.Tensor]:
        import torch.distributed as dist

        e, f = rank_contribution(self.pot, self.plan, self.rank, coordinates, species)
        if self.world > 1:
            ef = torch.cat([e.reshape(1), f.reshape(-1)])
            dist.all_reduce(ef, group=self.group)  # the exchange step: ghost forces reach their owners
            e, f = ef[0], ef[1:].reshape(-1, 3)
        return e, f
